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
    unsigned h;         // pairing bits: the gate qubits with position >= ls, or qubit ls alone
                        // when every gate qubit lies inside the sub-tile
    unsigned hb[3];     // their positions in segment-index space (q - ls), ascending
    unsigned k;         // gate qubits
    unsigned vbit[3];   // virtual-index bit of gate qubit j; j = 0 is the MSB of the local index
    idx_t nbase;        // base segments per dimension: (d >> ls) >> h
    idx_t items;        // nbase * (nbase + 1) / 2
    unsigned fixmask;   // bit l set: local index l is left in place with phase 1 by the gate
                        // (monomial gates only; an element whose row and column are both
                        // fixed is unchanged and is neither loaded nor stored)
    unsigned long long fixrows;  // the same as a mask over virtual indices (dm_fixed_rows)
    unsigned long long hcmask;   // controlled flips: control qubits above the sub-tile that are
                                 // not pairing bits (one value per item's rows or columns)
    unsigned long long wait_limit = 1ull << 24;   // polls of a bounded wait for staged data
    unsigned drop_loads = 0;     // test hook: arm the barrier but issue no copy, so the wait
                                 // for the item's data runs out (nothing is in flight)
    ORKAN_HD unsigned S() const { return 1u << ls; }
    ORKAN_HD unsigned V() const { return 1u << (ls + h); }
    ORKAN_HD unsigned P() const { return V() + 1; }    // smem row pitch (padded)
};

// Choose the sub-tile side: the largest S (<= 2^ls_max) whose block side V = S * 2^h stays
// within the cap: max_v_low when at most one gate qubit lies above the sub-tile, 64
// otherwise (keeping bulk-copy lines long when the block holds many sub-tiles).
// qubits[j] is gate qubit j, qubits[0] the most significant bit of the local index.
inline bool dm_geometry(unsigned n, unsigned k, const unsigned* qubits, unsigned ls_max, DmGeom* g,
                        unsigned max_v_low = kDmMaxV) {
    if (k < 1 || k > 3 || n < k) return false;
    for (unsigned j = 0; j < k; ++j) {
        if (qubits[j] >= n) return false;
        for (unsigned i = 0; i < j; ++i) if (qubits[i] == qubits[j]) return false;
    }
    unsigned ls = ls_max < n ? ls_max : n;
    for (;; --ls) {
        unsigned h = 0;
        for (unsigned j = 0; j < k; ++j) h += (qubits[j] >= ls);
        const unsigned long long cap = h <= 1 ? (unsigned long long)max_v_low * max_v_low : kDmMaxElems;
        if ((1ull << (2 * (ls + h))) <= cap || ls == 0) {
            // a gate that stays inside the sub-tile (h = 0) still pairs the sub-tiles along
            // qubit ls when the doubled block fits: four times fewer, four times larger items
            const bool widen = (h == 0 && ls < n && (1ull << (2 * (ls + 1))) <= cap);
            g->d = idx_t(1) << n;
            g->n = n;
            g->ls = ls;
            g->h = widen ? 1u : h;
            g->k = k;
            // high qubits in ascending order -> hb, and their virtual bits ls + rank
            unsigned hq[3], nh = 0;
            for (unsigned j = 0; j < k; ++j) if (qubits[j] >= ls) hq[nh++] = qubits[j];
            if (widen) hq[nh++] = ls;
            h = g->h;
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
            g->hcmask = 0;
            return true;
        }
        if (ls == 0) return false;
    }
}

// Sub-tile classes of position (a, b) of an item.
enum : int { kSubDirect = 0, kSubDiag = 1, kSubTransposed = 2, kSubSkip = 3 };

// ---------------------------------------------------------------------------------
// Staging.  The block is held in shared memory as vb[M * P + m] with M the "major" and
// m the "minor" virtual index: major = row for the tiled layout and column for the packed
// layout, so that a line of a stored sub-tile (a tile row / a packed column segment: S
// consecutive storage elements) lands on consecutive shared-memory addresses and moves
// with ONE bulk copy (TMA, cp.async.bulk).  For the packed layout the block therefore
// holds rho^T, and the gate parameters are transformed once on the host so that the same
// group operations compute (U rho U^dagger)^T = conj(U) rho^T conj(U)^dagger
// (dm_orient_* below).
//
// Region of position (a, b): major indices MB..MB+S, minor indices mB..mB+S; stored line
// `line`, offset p lands at (MB + line) * P + mB + p.  Regions needing more than a copy:
//   transposed position  its stored partner lands in stored orientation and is
//                        conjugate-transposed in place after the copy (and back before
//                        the store);
//   diagonal sub-tile    only the stored (lower) half lands; the other half is the
//                        conjugate transpose (for the tiled layout it is regenerated
//                        from the lower half again before the store, so diagonal tiles
//                        keep an exact mirror);
//   direct position of a diagonal item (has_c)
//                        its transposed position (b, a) is filled with the conjugate
//                        transpose of the region.
// ---------------------------------------------------------------------------------
struct DmPos {
    idx_t gbase;     // storage index of element (line 0, p 0) of the stored sub-tile
    idx_t mbase;     // tiled: storage index of the mirror of (line 0, p 0); written at mbase + p*T + line
    idx_t gcol;      // packed: d - PC - 1, the column-start increment per line
    int MB, mB;      // region origin in vb (major, minor)
    int cls;         // kSub*
    int has_c;       // direct sub-tile of a diagonal item: also fill the transposed region
    int mirror;      // tiled: the stored sub-tile lies in a diagonal tile, rewrite its mirror
    int fconst;      // virtual index constant along a line: fconst + line
    int fvar;        // virtual index varying along a line: fvar + p
    int allvar;      // every fvar + p (p < S) is a fixed row/column of the gate
    unsigned bytes;  // bytes this position's lines bring in (for the transaction count)
    int pad_;
    unsigned long long fmc;   // virtual indices fixed by the gate along the line-constant axis
    unsigned long long pad2_;
};
constexpr unsigned kDmMaxPos = 64;                     // 4^h with h <= 3
// One more descriptor slot after the positions holds the item's flags (cls field): bit 0
// the staged block's major, bit 1 its minor indices meet the high controls of a controlled
// flip (major = rows for the tiled layout, columns for the packed one); bit 2 the item is
// left unchanged (neither its rows nor its columns meet them) and is skipped.
constexpr unsigned kDmItemSlot = kDmMaxPos;
constexpr unsigned kDmPosBytes = (kDmMaxPos + 1) * sizeof(DmPos);
static_assert(sizeof(DmPos) == 80, "descriptor size");
static_assert(kDmPosBytes % 16 == 0, "descriptor block keeps the staged block 16-byte aligned");

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

// Line range [p0, p1) a stored line contributes (the lower half only on diagonal sub-tiles).
template <class Map>
ORKAN_HD void dm_line_range(const DmPos& q, unsigned line, unsigned S, unsigned* p0, unsigned* p1) {
    if (q.cls == kSubDiag) {
        if (Map::kRowContig) { *p0 = line; *p1 = S; }     // packed column: rows >= column
        else { *p0 = 0; *p1 = line + 1; }                  // tile row: columns <= row
    } else {
        *p0 = 0;
        *p1 = S;
    }
}

// A line every element of which the gate leaves in place: neither loaded nor stored.
ORKAN_HD bool dm_line_skipped(const DmPos& q, unsigned line) {
    return q.allvar && ((q.fmc >> (q.fconst + line)) & 1ull);
}

// Build the descriptors of item w (threads tid < 4^h, one position each).
template <class Map>
ORKAN_HD void dm_setup(const Map& map, const DmGeom& g, idx_t w, DmPos* pd, unsigned tid, unsigned nthr) {
    const unsigned h = g.h, ls = g.ls, S = g.S();
    const unsigned npos = 1u << (2 * h);
    if (tid >= npos) return;
    idx_t u, v;
    tri_unrank_f(w, &u, &v);
    const bool diag_item = (u == v);
    const idx_t rb = insert0_sorted(u, g.hb, h), cb = insert0_sorted(v, g.hb, h);
    // high controls of a controlled flip: one value for all rows (columns) of the item; rows
    // that do not meet them are all fixed
    const unsigned long long hc = g.hcmask;
    const bool rowc = ((unsigned long long)(rb << ls) & hc) == hc, colc = ((unsigned long long)(cb << ls) & hc) == hc;
    const unsigned V = g.V();
    const unsigned long long allv = V >= 64 ? ~0ull : ((1ull << V) - 1ull);
    const unsigned long long fm_row = rowc ? g.fixrows : allv, fm_col = colc ? g.fixrows : allv;
    const bool any_fixed = (fm_row | fm_col) != 0;
    if (tid == 0) {
        DmPos f{};
        const bool maj = Map::kRowContig ? colc : rowc, mnr = Map::kRowContig ? rowc : colc;
        f.cls = (maj ? 1 : 0) | (mnr ? 2 : 0) | ((!rowc && !colc) ? 4 : 0);
        pd[kDmItemSlot] = f;
    }
    const unsigned long long smask = (S >= 64) ? ~0ull : ((1ull << S) - 1ull);
    for (unsigned t = tid; t < npos; t += nthr) {
        const unsigned a = t >> h, b = t & ((1u << h) - 1);
        const idx_t R = (rb | spread_bits(a, g.hb, h)) << ls;
        const idx_t C = (cb | spread_bits(b, g.hb, h)) << ls;
        const int aS = (int)(a * S), bS = (int)(b * S);
        DmPos q;
        q.gbase = 0;
        q.mbase = 0;
        q.gcol = 0;
        q.has_c = 0;
        q.mirror = 0;
        q.pad_ = 0;
        q.pad2_ = 0;
        q.MB = Map::kRowContig ? bS : aS;
        q.mB = Map::kRowContig ? aS : bS;
        // virtual coordinates along a stored line: tiled line = virtual row (aS + line) for a
        // direct sub-tile; packed line = virtual column (bS + line); transposed: swapped
        const bool tr = (R < C);
        if (Map::kRowContig) { q.fconst = tr ? aS : bS; q.fvar = tr ? bS : aS; }
        else                 { q.fconst = tr ? bS : aS; q.fvar = tr ? aS : bS; }
        const bool const_is_row = Map::kRowContig ? tr : !tr;
        q.fmc = const_is_row ? fm_row : fm_col;
        const unsigned long long fm_var = const_is_row ? fm_col : fm_row;
        if (R > C) {
            q.cls = kSubDirect;
            q.gbase = map.at(R, C);
            q.has_c = diag_item ? 1 : 0;
            if (Map::kRowContig) q.gcol = map.d - C - 1;
            else if (map.same_storage_block(R, C)) { q.mirror = 1; q.mbase = map.at(C, R); }
        } else if (R == C) {
            q.cls = kSubDiag;
            q.gbase = map.at(R, R);
            if (Map::kRowContig) q.gcol = map.d - R - 1;
        } else if (!diag_item) {
            q.cls = kSubTransposed;
            q.gbase = map.at(C, R);                          // stored partner (C, R)
            if (Map::kRowContig) q.gcol = map.d - R - 1;
            else if (map.same_storage_block(C, R)) { q.mirror = 1; q.mbase = map.at(R, C); }
        } else {
            q.cls = kSubSkip;
        }
        // tiled diagonal sub-tiles are stored as whole rows whose upper half is rebuilt from
        // the lower half, so none of their rows may be skipped
        const bool no_skip = Map::kMirrors && q.cls == kSubDiag;
        q.allvar = (any_fixed && !no_skip && ((fm_var >> q.fvar) & smask) == smask) ? 1 : 0;
        // bytes the position's lines bring in: whole S x S sub-tile, or the lower half of a
        // diagonal one, less the lines skipped because every element in them is fixed
        unsigned bytes = 0;
        if (q.cls != kSubSkip) {
            const unsigned full = q.cls == kSubDiag ? S * (S + 1) / 2 : S * S;
            bytes = full * 16u;
            if (q.allvar) {
                const unsigned long long skip = (q.fmc >> q.fconst) & smask;
                if (q.cls != kSubDiag) {
                    bytes -= (unsigned)popc64(skip) * S * 16u;
                } else {                                   // packed diagonal: line j holds S - j
                    for (unsigned long long m = skip; m; m &= m - 1) bytes -= (S - ctz64(m)) * 16u;
                }
            }
        }
        q.bytes = bytes;
        pd[t] = q;
    }
}

// Storage index of element (line, p) of a position's stored sub-tile.
template <class Map>
ORKAN_HD idx_t dm_addr(const Map& map, const DmPos& q, unsigned line, unsigned p) {
    if (Map::kRowContig) return q.gbase + (idx_t)line * q.gcol - (idx_t)((line * (line - 1)) >> 1) + p;
    return q.gbase + ((idx_t)line << map.log_tdim()) + p;
}

// Bulk copies of one item: lines are numbered t = pos * S + line over all positions; the
// caller's threads take lines tid, tid + nthr, ...  Mem::bulk_load / bulk_store move
// (p1 - p0) consecutive elements.
template <class Map, class Mem>
ORKAN_HD void dm_bulk_loads(const Mem& mem, const Map& map, const DmGeom& g, const DmPos* pd, double2* vb,
                            void* bar, unsigned tid, unsigned nthr) {
    const unsigned ls = g.ls, S = g.S(), P = g.P();
    const unsigned nlines = 1u << (2 * g.h + ls);
    for (unsigned t = tid; t < nlines; t += nthr) {
        const DmPos& q = pd[t >> ls];
        const unsigned line = t & (S - 1);
        if (q.cls == kSubSkip || dm_line_skipped(q, line)) continue;
        unsigned p0, p1;
        dm_line_range<Map>(q, line, S, &p0, &p1);
        mem.bulk_load(vb + (q.MB + (int)line) * (int)P + q.mB + (int)p0, dm_addr(map, q, line, p0), p1 - p0, bar);
    }
}

template <class Map, class Mem>
ORKAN_HD void dm_bulk_stores(const Mem& mem, const Map& map, const DmGeom& g, const DmPos* pd, const double2* vb,
                             unsigned tid, unsigned nthr) {
    const unsigned ls = g.ls, S = g.S(), P = g.P();
    const unsigned nlines = 1u << (2 * g.h + ls);
    for (unsigned t = tid; t < nlines; t += nthr) {
        const DmPos& q = pd[t >> ls];
        const unsigned line = t & (S - 1);
        if (q.cls == kSubSkip || dm_line_skipped(q, line)) continue;
        unsigned p0 = 0, p1 = S;                            // tiled diagonal tiles: whole rows
        if (Map::kRowContig) dm_line_range<Map>(q, line, S, &p0, &p1);
        mem.bulk_store(dm_addr(map, q, line, p0), vb + (q.MB + (int)line) * (int)P + q.mB + (int)p0, p1 - p0);
    }
}

// Does position q need work in pass `kind` (0: after the copies land, 1: before the store,
// 2: per-element mirror stores)?
template <class Map>
ORKAN_HD bool dm_needs(const DmPos& q, int kind) {
    if (kind == 2) return Map::kMirrors && q.mirror;
    if (q.cls == kSubTransposed) return true;
    if (q.cls == kSubDiag) return kind == 0 || Map::kMirrors;
    return kind == 0 && q.cls == kSubDirect && q.has_c;
}

// Bit mask over the item's positions of those needing pass `kind`.
template <class Map>
ORKAN_HD unsigned long long dm_pass_mask(const DmPos* pd, unsigned npos, int kind) {
#ifdef __CUDA_ARCH__
    const unsigned lane = threadIdx.x & 31u;
    const unsigned lo = __ballot_sync(0xffffffffu, lane < npos && dm_needs<Map>(pd[lane], kind));
    const unsigned hi = __ballot_sync(0xffffffffu, lane + 32 < npos && dm_needs<Map>(pd[lane + 32], kind));
    return (unsigned long long)lo | ((unsigned long long)hi << 32);
#else
    unsigned long long m = 0;
    for (unsigned t = 0; t < npos; ++t)
        if (dm_needs<Map>(pd[t], kind)) m |= 1ull << t;
    return m;
#endif
}

// Tiled layout, sub-tiles smaller than a tile inside a diagonal tile: the mirror image of a
// stored element (line, p) is at mbase + p*T + line and holds its conjugate (per element,
// strided; occurs only when S < tile side).
template <class Map, class Mem>
ORKAN_HD void dm_mirror_stores(const Mem& mem, const Map& map, const DmGeom& g, const DmPos* pd,
                               const double2* vb, unsigned long long mask, unsigned tid, unsigned nthr) {
    if (!Map::kMirrors) return;
    const unsigned ls = g.ls, S = g.S(), P = g.P();
    while (mask) {
        const unsigned t = ctz64(mask);
        mask &= mask - 1;
        const DmPos& q = pd[t];
        for (unsigned e = tid; e < (1u << (2 * ls)); e += nthr) {
            const unsigned line = e >> ls, p = e & (S - 1);
            if (dm_line_skipped(q, line)) continue;
            mem.st(q.mbase + ((idx_t)p << map.log_tdim()) + line,
                   cconj(vb[(q.MB + (int)line) * (int)P + q.mB + (int)p]));
        }
    }
}

// In-place region fix-ups of the positions in `mask` (pairs (x, y) of a region handled by
// one thread each).  kind 0: after the copies land;  kind 1: before the store.
template <class Map>
ORKAN_HD void dm_fixups(const DmGeom& g, const DmPos* pd, double2* vb, int kind, unsigned long long mask,
                        unsigned tid, unsigned nthr) {
    const unsigned ls = g.ls, S = g.S(), P = g.P();
    while (mask) {
        const unsigned t = ctz64(mask);
        mask &= mask - 1;
        const DmPos& q = pd[t];
        double2* r = vb + q.MB * (int)P + q.mB;
        for (unsigned e = tid; e < (1u << (2 * ls)); e += nthr) {
            const unsigned x = e >> ls, y = e & (S - 1);
            if (q.cls == kSubTransposed) {
                // conjugate transpose in place: (x, y) <-> (y, x)
                if (x > y) continue;
                const double2 a = r[x * P + y];
                if (x == y) { r[x * P + y] = cconj(a); continue; }
                const double2 b = r[y * P + x];
                r[x * P + y] = cconj(b);
                r[y * P + x] = cconj(a);
            } else if (q.cls == kSubDiag) {
                // fill the half that was not copied from the half that was
                const bool landed = Map::kRowContig ? (y >= x) : (y <= x);
                if (!landed) r[x * P + y] = cconj(r[y * P + x]);
            } else {
                // direct sub-tile of a diagonal item: its transposed position (major mB.., minor MB..)
                vb[(q.mB + (int)y) * (int)P + q.MB + (int)x] = cconj(r[x * P + y]);
            }
        }
    }
}

// ---------------------------------------------------------------------------------
// Group operations on the staged block (vb[M * P + m]).  Each thread owns whole groups,
// so compute needs no synchronisation between threads.
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
// Bank-conflict-free order of a 2 x 2 group's two columns.  The lanes of a warp share the
// group row and take consecutive column indices with the gate bit inserted; for a gate bit
// below 3 the 8 lanes of a quarter warp then fall on only four 16-byte bank groups (every
// other slot).  Lanes with bit 2 set touch their second column first, which lies on the four
// other bank groups, so each access instruction of the quarter warp hits eight.
ORKAN_HD bool dm_swap_cols(unsigned vbq, unsigned lh, unsigned tid) { return vbq < 3 && lh >= 5 && (tid & 4u); }

struct OpMix1 {
    double2 u[4];
    ORKAN_HD void operator()(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr, unsigned = 3u) const {
        const unsigned P = g.P(), lh = g.ls + g.h - 1, vbq = g.vbit[0];
        const unsigned groups = 1u << (2 * lh);
        const bool sw = dm_swap_cols(vbq, lh, tid);
        for (unsigned t = tid; t < groups; t += nthr) {
            const unsigned r0 = (unsigned)insert0(t >> lh, vbq), c0 = (unsigned)insert0(t & ((1u << lh) - 1), vbq);
            const unsigned r1 = r0 | (1u << vbq), c1 = c0 | (1u << vbq);
            const unsigned ca = sw ? c1 : c0, cb = sw ? c0 : c1;
            const double2 y0a = vb[r0 * P + ca], y0b = vb[r0 * P + cb];
            const double2 y1a = vb[r1 * P + ca], y1b = vb[r1 * P + cb];
            const double2 x00 = sw ? y0b : y0a, x01 = sw ? y0a : y0b;
            const double2 x10 = sw ? y1b : y1a, x11 = sw ? y1a : y1b;
            // rows: Y = U X
            const double2 y00 = cadd(cmul(u[0], x00), cmul(u[1], x10));
            const double2 y01 = cadd(cmul(u[0], x01), cmul(u[1], x11));
            const double2 y10 = cadd(cmul(u[2], x00), cmul(u[3], x10));
            const double2 y11 = cadd(cmul(u[2], x01), cmul(u[3], x11));
            // columns: Z = Y U^dagger, Z[i][j] = sum_m Y[i][m] conj(U[j][m])
            const double2 z00 = cadd(cmulc(y00, u[0]), cmulc(y01, u[1]));
            const double2 z01 = cadd(cmulc(y00, u[2]), cmulc(y01, u[3]));
            const double2 z10 = cadd(cmulc(y10, u[0]), cmulc(y11, u[1]));
            const double2 z11 = cadd(cmulc(y10, u[2]), cmulc(y11, u[3]));
            vb[r0 * P + ca] = sw ? z01 : z00;
            vb[r0 * P + cb] = sw ? z00 : z01;
            vb[r1 * P + ca] = sw ? z11 : z10;
            vb[r1 * P + cb] = sw ? z10 : z11;
        }
    }
};

// Dense 2-qubit unitary U (row-major u[4*r + c], local index = 2*bit(q0) + bit(q1)).
struct OpMix2 {
    double2 u[16];
    ORKAN_HD void operator()(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr, unsigned = 3u) const {
        const unsigned P = g.P(), lq = g.ls + g.h - 2;
        unsigned asc[2] = {g.vbit[0] < g.vbit[1] ? g.vbit[0] : g.vbit[1],
                           g.vbit[0] < g.vbit[1] ? g.vbit[1] : g.vbit[0]};
        const unsigned groups = 1u << (2 * lq);
        for (unsigned t = tid; t < groups; t += nthr) {
            const unsigned rb = (unsigned)insert0_sorted(t >> lq, asc, 2);
            const unsigned cb = (unsigned)insert0_sorted(t & ((1u << lq) - 1), asc, 2);
            unsigned ri[4], ci[4];
            for (unsigned l = 0; l < 4; ++l) {
                ri[l] = dm_set_local(rb, l, g.vbit, 2);
                ci[l] = dm_set_local(cb, l, g.vbit, 2);
            }
            // the group's 16 elements belong to this thread alone: Y = U X column by column in
            // place, then Z = Y U^dagger row by row (few values live at a time)
            for (unsigned c = 0; c < 4; ++c) {
                double2 x[4];
                for (unsigned m = 0; m < 4; ++m) x[m] = vb[ri[m] * P + ci[c]];
                for (unsigned r = 0; r < 4; ++r) {
                    double2 acc = c2(0.0, 0.0);
                    for (unsigned m = 0; m < 4; ++m) acc = cadd(acc, cmul(u[4 * r + m], x[m]));
                    vb[ri[r] * P + ci[c]] = acc;
                }
            }
            for (unsigned r = 0; r < 4; ++r) {
                double2 y[4];
                for (unsigned m = 0; m < 4; ++m) y[m] = vb[ri[r] * P + ci[m]];
                for (unsigned c = 0; c < 4; ++c) {
                    double2 acc = c2(0.0, 0.0);
                    for (unsigned m = 0; m < 4; ++m) acc = cadd(acc, cmulc(y[m], u[4 * c + m]));
                    vb[ri[r] * P + ci[c]] = acc;
                }
            }
        }
    }
};

// 1-qubit superoperator (row-major s[4*m + j]) on vec = (x00, x01, x10, x11).
struct OpSuper1 {
    double2 s[16];
    ORKAN_HD void operator()(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr, unsigned = 3u) const {
        const unsigned P = g.P(), lh = g.ls + g.h - 1, vbq = g.vbit[0];
        const unsigned groups = 1u << (2 * lh);
        const bool sw = dm_swap_cols(vbq, lh, tid);
        for (unsigned t = tid; t < groups; t += nthr) {
            const unsigned r0 = (unsigned)insert0(t >> lh, vbq), c0 = (unsigned)insert0(t & ((1u << lh) - 1), vbq);
            const unsigned r1 = r0 | (1u << vbq), c1 = c0 | (1u << vbq);
            // the column order of each row as in OpMix1 (dm_swap_cols)
            const unsigned ca = sw ? c1 : c0, cb = sw ? c0 : c1;
            const double2 y0a = vb[r0 * P + ca], y0b = vb[r0 * P + cb];
            const double2 y1a = vb[r1 * P + ca], y1b = vb[r1 * P + cb];
            const double2 x[4] = {sw ? y0b : y0a, sw ? y0a : y0b, sw ? y1b : y1a, sw ? y1a : y1b};
            double2 out[4];
            for (unsigned m = 0; m < 4; ++m) {
                double2 acc = c2(0.0, 0.0);
                for (unsigned j = 0; j < 4; ++j) {          // four FMAs per complex term
                    const double2 sj = s[4 * m + j];
                    acc.x = fma(sj.x, x[j].x, acc.x);
                    acc.x = fma(-sj.y, x[j].y, acc.x);
                    acc.y = fma(sj.x, x[j].y, acc.y);
                    acc.y = fma(sj.y, x[j].x, acc.y);
                }
                out[m] = acc;
            }
            vb[r0 * P + ca] = sw ? out[1] : out[0];
            vb[r0 * P + cb] = sw ? out[0] : out[1];
            vb[r1 * P + ca] = sw ? out[3] : out[2];
            vb[r1 * P + cb] = sw ? out[2] : out[3];
        }
    }
};

// FP64 tensor-core form of the 2-qubit superoperator.  The update of one 4 x 4 group is a real
// 32 x 32 matrix A (rows: re / im of the 16 outputs; columns: re / im of the 16 inputs) times
// the group's 32 real inputs; a warp applies it to 8 groups at a time with 4 x 8 steps of
// mma.sync.m8n8k4.f64 (D = A B + D on 8 x 8 x 4; lane l holds A[l / 4][l % 4], B[l % 4][l / 4]
// and D[l / 4][2 (l % 4) + i], i = 0, 1).  Row tile mt (0 .. 3) of A holds output
// o = 8 (mt & 1) + l / 4, real part for mt < 2, imaginary part otherwise; k-step ks (0 .. 7)
// holds input j = 4 (ks & 3) + l % 4, real part for ks < 4; the columns of B are the 8 groups.
// One warp instruction does 256 FMA instead of 32, which leaves the issue slots to the loads,
// stores and index arithmetic around it.

// Staged index of the base element (local row 0, local column 0) of group t: the row and
// column parts of t with zeros inserted at the gate bits asc[0] < asc[1] (32-bit arithmetic).
ORKAN_HD unsigned super2_group_base(unsigned P, const unsigned* asc, unsigned lq, unsigned t) {
    unsigned r = t >> lq, c = t & ((1u << lq) - 1);
    for (unsigned j = 0; j < 2; ++j) {
        const unsigned lo = (1u << asc[j]) - 1;
        r = ((r & ~lo) << 1) | (r & lo);
        c = ((c & ~lo) << 1) | (c & lo);
    }
    return r * P + c;
}

// A lane's element offsets from a group's base element (the base has zeros at the gate bits,
// so an element is base + offset): in[r] for its inputs (local row r, local column lane % 4 of
// group base + lane / 4), out[h] for its outputs (local row 2 h + lane / 16, local column
// (lane / 4) % 4 of groups base + 2 (lane % 4) + i, i = 0, 1).
struct Super2Lane {
    unsigned in[4];
    unsigned out[2];
};
ORKAN_HD Super2Lane super2_lane(const DmGeom& g, unsigned lane) {
    Super2Lane L;
    const unsigned P = g.P(), gq = lane >> 2, q = lane & 3u;
    for (unsigned r = 0; r < 4; ++r) L.in[r] = dm_set_local(0u, r, g.vbit, 2) * P + dm_set_local(0u, q, g.vbit, 2);
    for (unsigned h = 0; h < 2; ++h)
        L.out[h] = dm_set_local(0u, 2 * h + (gq >> 2), g.vbit, 2) * P + dm_set_local(0u, gq & 3u, g.vbit, 2);
    return L;
}

// Lane's entry of A for row tile mt and k-step ks (superoperator sp, row-major 16 x 16).
ORKAN_HD double super2_afrag(const double2* sp, unsigned mt, unsigned ks, unsigned lane) {
    const unsigned o = 8 * (mt & 1) + (lane >> 2), j = 4 * (ks & 3) + (lane & 3);
    const double2 e = sp[16 * o + j];
    const bool re_out = mt < 2, re_in = ks < 4;
    // re out = sum (e.re x.re - e.im x.im), im out = sum (e.im x.re + e.re x.im)
    return re_out == re_in ? e.x : (re_out ? -e.y : e.y);
}

#ifdef __CUDACC__
__device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
        : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}
#endif

// A fragments of one lane (built once per engine block).
struct Super2Frag {
    double a[4][8];
};

// Whether an item of geometry g takes the tensor-core form (8 groups per warp step).  Then
// the staged block has V >= 16 rows of P = V + 1 slots, at least 272, so it can hold the 256
// superoperator entries while the fragments are built (dm_op_prepare).
ORKAN_HD bool super2_mma_form(const DmGeom& g, unsigned nthr) {
    return g.ls + g.h >= 4 && (nthr & 31u) == 0;
}
ORKAN_HD bool super2_stage_fits(const DmGeom& g) { return (unsigned long long)g.V() * g.P() >= 256ull; }

// 2-qubit superoperator (row-major s[16 * m + j], vec index 4 * row + column of the 4 x 4
// block over the two gate qubits, local index 2 * bit(q0) + bit(q1)) on 4 x 4 groups.
struct OpSuper2 {
    double2 s[256];
#ifdef __CUDACC__
    // Tensor-core form of one item with the lane's fragments f: warp w takes groups
    // 8 w .. 8 w + 7, then 8 (w + warps) ...; the mma of a warp reads every lane's inputs
    // before any lane stores, and the groups of different warps are disjoint.
    __device__ void mma_groups(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr, const Super2Frag& f) const {
        const unsigned P = g.P(), lq = g.ls + g.h - 2;
        unsigned asc[2] = {g.vbit[0] < g.vbit[1] ? g.vbit[0] : g.vbit[1],
                           g.vbit[0] < g.vbit[1] ? g.vbit[1] : g.vbit[0]};
        const unsigned groups = 1u << (2 * lq);
        const unsigned lane = tid & 31u, gq = lane >> 2, q = lane & 3u;
        const double(&a)[4][8] = f.a;
        const Super2Lane L = super2_lane(g, lane);
        for (unsigned base = 8 * (tid >> 5); base < groups; base += 8 * (nthr >> 5)) {
            const unsigned ein = super2_group_base(P, asc, lq, base + gq);
            double b[8];
#pragma unroll
            for (unsigned r = 0; r < 4; ++r) {
                const double2 x = vb[ein + L.in[r]];
                b[r] = x.x;
                b[r + 4] = x.y;
            }
            double d[4][2];
#pragma unroll
            for (unsigned mt = 0; mt < 4; ++mt) {
                d[mt][0] = 0.0;
                d[mt][1] = 0.0;
#pragma unroll
                for (unsigned ks = 0; ks < 8; ++ks) dmma_884(d[mt][0], d[mt][1], a[mt][ks], b[ks]);
            }
#pragma unroll
            for (unsigned i = 0; i < 2; ++i) {
                const unsigned eout = super2_group_base(P, asc, lq, base + 2 * q + i);
                vb[eout + L.out[0]] = c2(d[0][i], d[2][i]);
                vb[eout + L.out[1]] = c2(d[1][i], d[3][i]);
            }
        }
    }
#endif

    // Scalar form (items of fewer than 8 groups), and on the host also the tensor-core form,
    // carried out by lane 0 of each warp with the fragment layout of the instruction.
    ORKAN_HD void operator()(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr, unsigned = 3u) const {
        const double2* sp = s;     // read in the same order by every thread: broadcast loads
        const unsigned P = g.P(), lq = g.ls + g.h - 2;
        unsigned asc[2] = {g.vbit[0] < g.vbit[1] ? g.vbit[0] : g.vbit[1],
                           g.vbit[0] < g.vbit[1] ? g.vbit[1] : g.vbit[0]};
        const unsigned groups = 1u << (2 * lq);
#ifndef __CUDA_ARCH__
        if (super2_mma_form(g, nthr) && super2_stage_fits(g)) {
            // host: lane 0 of each warp carries out the warp's steps with the fragment layout
            // of the instruction, through the same index and fragment functions
            if (tid & 31u) return;
            for (unsigned base = 8 * (tid >> 5); base < groups; base += 8 * (nthr >> 5)) {
                double b[32][8], d[32][4][2];
                for (unsigned l = 0; l < 32; ++l) {
                    const Super2Lane L = super2_lane(g, l);
                    const unsigned ein = super2_group_base(P, asc, lq, base + (l >> 2));
                    for (unsigned r = 0; r < 4; ++r) {
                        const double2 x = vb[ein + L.in[r]];
                        b[l][r] = x.x;
                        b[l][r + 4] = x.y;
                    }
                }
                for (unsigned mt = 0; mt < 4; ++mt) {
                    double D[8][8] = {};
                    for (unsigned ks = 0; ks < 8; ++ks)
                        for (unsigned m = 0; m < 8; ++m)
                            for (unsigned nn = 0; nn < 8; ++nn)
                                for (unsigned k = 0; k < 4; ++k)
                                    D[m][nn] = fma(super2_afrag(sp, mt, ks, 4 * m + k), b[4 * nn + k][ks], D[m][nn]);
                    for (unsigned l = 0; l < 32; ++l)
                        for (unsigned i = 0; i < 2; ++i) d[l][mt][i] = D[l >> 2][2 * (l & 3u) + i];
                }
                for (unsigned l = 0; l < 32; ++l) {
                    const Super2Lane L = super2_lane(g, l);
                    for (unsigned i = 0; i < 2; ++i) {
                        const unsigned eout = super2_group_base(P, asc, lq, base + 2 * (l & 3u) + i);
                        vb[eout + L.out[0]] = c2(d[l][0][i], d[l][2][i]);
                        vb[eout + L.out[1]] = c2(d[l][1][i], d[l][3][i]);
                    }
                }
            }
            return;
        }
#endif
        for (unsigned t = tid; t < groups; t += nthr) {
            const unsigned rb = (unsigned)insert0_sorted(t >> lq, asc, 2);
            const unsigned cb = (unsigned)insert0_sorted(t & ((1u << lq) - 1), asc, 2);
            unsigned ri[4], ci[4];
            for (unsigned l = 0; l < 4; ++l) {
                ri[l] = dm_set_local(rb, l, g.vbit, 2);
                ci[l] = dm_set_local(cb, l, g.vbit, 2);
            }
            // the group's 16 elements belong to this thread alone: all read, then written
            double2 x[16];
            for (unsigned r = 0; r < 4; ++r)
                for (unsigned c = 0; c < 4; ++c) x[4 * r + c] = vb[ri[r] * P + ci[c]];
#pragma unroll 1
            for (unsigned r = 0; r < 4; ++r) {                // output row r, two outputs at a time
                const unsigned rowoff = dm_set_local(rb, r, g.vbit, 2) * P;
#pragma unroll
                for (unsigned c = 0; c < 4; c += 2) {
                    const unsigned m = 4 * r + c;
                    double2 acc0 = c2(0.0, 0.0), acc1 = c2(0.0, 0.0);
                    // complex multiply-add as four FMAs (a product then an add would take six
                    // FP64 operations per term)
#pragma unroll
                    for (unsigned j = 0; j < 16; ++j) {
                        const double2 s0 = sp[16 * m + j], s1 = sp[16 * m + 16 + j];
                        acc0.x = fma(s0.x, x[j].x, acc0.x);
                        acc0.x = fma(-s0.y, x[j].y, acc0.x);
                        acc0.y = fma(s0.x, x[j].y, acc0.y);
                        acc0.y = fma(s0.y, x[j].x, acc0.y);
                        acc1.x = fma(s1.x, x[j].x, acc1.x);
                        acc1.x = fma(-s1.y, x[j].y, acc1.x);
                        acc1.y = fma(s1.x, x[j].y, acc1.y);
                        acc1.y = fma(s1.y, x[j].x, acc1.y);
                    }
                    vb[rowoff + ci[c]] = acc0;
                    vb[rowoff + ci[c + 1]] = acc1;
                }
            }
        }
    }
};

// Monomial gate U|x> with an involutive permutation (X, Y, CX, CY, SWAP, CCX ...):
// (U psi)[y] = phase[y] * psi[src[y]] on the local index, src[src[y]] == y.
// Element pairs (y, z) <-> (src y, src z) are 2-cycles; the thread owning the
// smaller flat index of a pair updates both.
// The gates of the library are controlled flips: on virtual indices the image of x is
// x ^ tmask when cond(x) holds -- all bits of cmask set (X, Y, CX, CY, CCX), or the two
// bits of tmask different (SWAP) -- with phase p1 / p0 (target bit of x set / clear) where
// it holds and 1 elsewhere.  dm_monomial_tables recognises that form (flip = 1) and the
// operator then needs a few bit operations per element; other involutions use the local
// index tables src / phase.
struct OpMonomial {
    unsigned src[8];
    double2 phase[8];
    int flip;              // 1: controlled-flip form below
    int parity;            // cond(x): 0 all cmask bits set, 1 the two tmask bits differ
    unsigned cmask, tmask, tbit;
    double2 p0, p1;
    ORKAN_HD unsigned image(unsigned x, const DmGeom& g, double2* ph) const {
        if (flip) {
            const bool c = parity ? (((x & tmask) != 0) && ((x & tmask) != tmask)) : ((x & cmask) == cmask);
            *ph = c ? ((x & tbit) ? p1 : p0) : c2(1.0, 0.0);
            return c ? x ^ tmask : x;
        }
        const unsigned l = dm_get_local(x, g.vbit, g.k);
        *ph = phase[l];
        return dm_set_local(x, src[l], g.vbit, g.k);
    }
    ORKAN_HD void operator()(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr, unsigned iflags = 3u) const {
        if (flip && !parity) { flip_groups(g, vb, tid, nthr, iflags); return; }
        if (flip) { swap_groups(g, vb, tid, nthr); return; }
        const unsigned V = g.V(), P = g.P(), lv = g.ls + g.h;
        const unsigned total = V * V;
        for (unsigned f = tid; f < total; f += nthr) {
            const unsigned r = f >> lv, c = f & (V - 1);
            double2 pr, pc;
            const unsigned r2 = image(r, g, &pr), c2i = image(c, g, &pc);
            const unsigned f2 = (r2 << lv) + c2i;
            if (f2 < f) continue;
            const double2 fa = cmulc(pr, pc);
            if (f2 == f) {
                vb[r * P + c] = cmul(fa, vb[r * P + c]);
            } else {
                double2 pr2, pc2;
                image(r2, g, &pr2);
                image(c2i, g, &pc2);
                const double2 fb = cmulc(pr2, pc2);
                const double2 va = vb[r * P + c], vb2 = vb[r2 * P + c2i];
                vb[r * P + c] = cmul(fa, vb2);
                vb[r2 * P + c2i] = cmul(fb, va);
            }
        }
    }
    // Controlled flips: 2 x 2 groups over the target bit.  The control bits are the same for
    // both rows (columns) of a group, so the rows are exchanged (with phases p0, p1) when the
    // rows satisfy the condition, the columns likewise; groups where neither does are left
    // untouched (not read, not written).
    ORKAN_HD void flip_groups(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr, unsigned iflags) const {
        const bool rowc = iflags & 1u, colc = (iflags >> 1) & 1u;     // high controls (major, minor)
        const unsigned P = g.P(), lh = g.ls + g.h - 1, tpos = ctz64(tmask);
        const unsigned groups = 1u << (2 * lh);
        const double2 one = c2(1.0, 0.0);
        for (unsigned t = tid; t < groups; t += nthr) {
            const unsigned r0 = (unsigned)insert0(t >> lh, tpos), c0 = (unsigned)insert0(t & ((1u << lh) - 1), tpos);
            const bool cr = rowc && (r0 & cmask) == cmask, cc = colc && (c0 & cmask) == cmask;
            if (!cr && !cc) continue;
            const unsigned r1 = r0 | tmask, c1 = c0 | tmask;
            const double2 x00 = vb[r0 * P + c0], x01 = vb[r0 * P + c1];
            const double2 x10 = vb[r1 * P + c0], x11 = vb[r1 * P + c1];
            // row phases (target bit 0 / 1 of the new row) and column phases
            const double2 pr0 = cr ? p0 : one, pr1 = cr ? p1 : one, pc0 = cc ? p0 : one, pc1 = cc ? p1 : one;
            const double2 s00 = cr ? (cc ? x11 : x10) : (cc ? x01 : x00);
            const double2 s01 = cr ? (cc ? x10 : x11) : (cc ? x00 : x01);
            const double2 s10 = cr ? (cc ? x01 : x00) : (cc ? x11 : x10);
            const double2 s11 = cr ? (cc ? x00 : x01) : (cc ? x10 : x11);
            vb[r0 * P + c0] = cmul(cmulc(pr0, pc0), s00);
            vb[r0 * P + c1] = cmul(cmulc(pr0, pc1), s01);
            vb[r1 * P + c0] = cmul(cmulc(pr1, pc0), s10);
            vb[r1 * P + c1] = cmul(cmulc(pr1, pc1), s11);
        }
    }
    // SWAP: 4 x 4 groups over the two bits (index order 00, a, b, ab); rows and columns a <-> b.
    ORKAN_HD void swap_groups(const DmGeom& g, double2* vb, unsigned tid, unsigned nthr) const {
        const unsigned P = g.P(), lq = g.ls + g.h - 2;
        const unsigned lo = tmask & (0u - tmask), hi = tmask ^ lo;
        const unsigned asc[2] = {(unsigned)ctz64(lo), (unsigned)ctz64(hi)};
        const unsigned groups = 1u << (2 * lq);
        const unsigned sg[4] = {0, 2, 1, 3};                  // 00, lo, hi, both -> image
        for (unsigned t = tid; t < groups; t += nthr) {
            const unsigned rb = (unsigned)insert0_sorted(t >> lq, asc, 2);
            const unsigned cb = (unsigned)insert0_sorted(t & ((1u << lq) - 1), asc, 2);
            const unsigned off[4] = {0, lo, hi, lo | hi};
            double2 x[4][4];
            for (unsigned i = 0; i < 4; ++i)
                for (unsigned j = 0; j < 4; ++j) x[i][j] = vb[(rb | off[i]) * P + (cb | off[j])];
            for (unsigned i = 0; i < 4; ++i)
                for (unsigned j = 0; j < 4; ++j)
                    if (sg[i] != i || sg[j] != j) vb[(rb | off[i]) * P + (cb | off[j])] = x[sg[i]][sg[j]];
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

// Controlled-flip form of a k-qubit monomial gate: the last gate qubit (local bit 0) is the
// target, the others are controls; local index l goes to l ^ 1 when every control bit is set
// and stays in place with phase 1 otherwise (X, Y, CX, CY, CCX).
inline bool monomial_is_controlled_flip(const OpMonomial& op, unsigned k) {
    const unsigned m = 1u << k;
    for (unsigned l = 0; l < m; ++l) {
        const bool on = (l | 1u) == m - 1;                       // every control bit set
        if (op.src[l] != (on ? (l ^ 1u) : l)) return false;
        if (!on && !(op.phase[l].x == 1.0 && op.phase[l].y == 0.0)) return false;
    }
    return true;
}

// Host set-up of a monomial gate launch (geometry, fixed rows, operator form).
//
// A controlled flip is laid out over its target alone, so its block is as small as a
// 1-qubit gate's: a control inside the block (below the sub-tile or on a pairing bit)
// becomes a virtual-index condition (cmask), a control above it a condition on the item's
// rows and columns (hcmask), and items that meet it in neither are skipped.  A SWAP with
// unit phases uses the parity form; other gates the generic table over all their qubits.
inline bool dm_monomial_setup(unsigned n, unsigned k, const unsigned* qubits, OpMonomial& op, unsigned ls_max,
                              unsigned max_v_low, DmGeom* g) {
    const unsigned m = 1u << k;
    op.flip = 0;
    op.parity = 0;
    op.cmask = op.tmask = op.tbit = 0;
    op.p0 = op.p1 = c2(1.0, 0.0);
    if (k < 1 || k > 3) return false;
    for (unsigned j = 0; j < k; ++j) {
        if (qubits[j] >= n) return false;
        for (unsigned i = 0; i < j; ++i) if (qubits[i] == qubits[j]) return false;
    }
    if (monomial_is_controlled_flip(op, k)) {
        if (!dm_geometry(n, 1, &qubits[k - 1], ls_max, g, max_v_low)) return false;
        op.flip = 1;
        op.tmask = op.tbit = 1u << g->vbit[0];
        op.p0 = op.phase[m - 2];
        op.p1 = op.phase[m - 1];
        for (unsigned j = 0; j + 1 < k; ++j) {
            const unsigned q = qubits[j];
            if (q < g->ls) { op.cmask |= 1u << q; continue; }
            unsigned r = 0;
            while (r < g->h && g->hb[r] != q - g->ls) ++r;
            if (r < g->h) op.cmask |= 1u << (g->ls + r);           // a pairing bit of the block
            else g->hcmask |= 1ull << q;
        }
        unsigned long long fr = 0;
        if (op.cmask)
            for (unsigned x = 0; x < g->V(); ++x)
                if ((x & op.cmask) != op.cmask) fr |= 1ull << x;
        g->fixrows = fr;
        return true;
    }
    if (!dm_geometry(n, k, qubits, ls_max, g, max_v_low)) return false;
    g->fixmask = monomial_fixmask(op, m);
    g->fixrows = dm_fixed_rows(*g);
    if (k == 2 && op.src[0] == 0 && op.src[1] == 2 && op.src[2] == 1 && op.src[3] == 3) {
        bool unit = true;
        for (unsigned l = 0; l < 4; ++l) unit = unit && op.phase[l].x == 1.0 && op.phase[l].y == 0.0;
        if (unit) {
            op.flip = 1;
            op.parity = 1;
            op.tmask = (1u << g->vbit[0]) | (1u << g->vbit[1]);
            op.tbit = 1u << g->vbit[1];
        }
    }
    return true;
}

// The packed layout stages rho^T: (U rho U^dagger)^T = conj(U) rho^T conj(U)^dagger, so its
// operators are the complex conjugates; a superoperator on vec(rho_2x2) = (00, 01, 10, 11)
// acts on vec(rho^T) with 01 and 10 exchanged in both its rows and its columns.
inline void dm_orient(OpMix1& op, bool transposed) {
    if (transposed) for (auto& z : op.u) z = cconj(z);
}
inline void dm_orient(OpMix2& op, bool transposed) {
    if (transposed) for (auto& z : op.u) z = cconj(z);
}
inline void dm_orient(OpMonomial& op, bool transposed) {
    if (!transposed) return;
    for (auto& z : op.phase) z = cconj(z);
    op.p0 = cconj(op.p0);
    op.p1 = cconj(op.p1);
}
// vec(rho^T) holds element (i, j) at 4 j + i: rows and columns of the superoperator are
// permuted by 4 i + j <-> 4 j + i.
inline void dm_orient(OpSuper2& op, bool transposed) {
    if (!transposed) return;
    double2 t[256];
    for (unsigned m = 0; m < 16; ++m)
        for (unsigned j = 0; j < 16; ++j) t[16 * m + j] = op.s[16 * (((m & 3) << 2) | (m >> 2)) + (((j & 3) << 2) | (j >> 2))];
    for (unsigned i = 0; i < 256; ++i) op.s[i] = t[i];
}
inline void dm_orient(OpSuper1& op, bool transposed) {
    if (!transposed) return;
    const unsigned perm[4] = {0, 2, 1, 3};
    double2 t[16];
    for (unsigned m = 0; m < 4; ++m)
        for (unsigned j = 0; j < 4; ++j) t[4 * m + j] = op.s[4 * perm[m] + perm[j]];
    for (unsigned i = 0; i < 16; ++i) op.s[i] = t[i];
}

// Shared memory of one engine block: the mbarrier, the descriptors, the staged block.
ORKAN_HD size_t dm_stage_bytes(const DmGeom& g) { return kDmPosBytes + (size_t)g.V() * g.P() * 16; }
ORKAN_HD size_t dm_block_smem_bytes(const DmGeom& g) { return 16 + dm_stage_bytes(g); }

// One work item, phase by phase (the CPU emulator runs each phase for all threads before
// the next; k_dm_engine runs the same phases with block barriers between them).
template <class Map, class Mem, class Op>
ORKAN_HD void dm_engine_item_phase(int phase, const Mem& mem, const Map& map, const DmGeom& g, const Op& op,
                                   idx_t w, DmPos* pd, double2* vb, unsigned tid, unsigned nthr) {
    const unsigned npos = 1u << (2 * g.h);
    if (phase > 0 && (pd[kDmItemSlot].cls & 4)) return;     // item left unchanged
    switch (phase) {
        case 0: dm_setup(map, g, w, pd, tid, nthr); break;
        case 1: dm_bulk_loads(mem, map, g, pd, vb, nullptr, tid, nthr); break;
        case 2: dm_fixups<Map>(g, pd, vb, 0, dm_pass_mask<Map>(pd, npos, 0), tid, nthr); break;
        case 3: op(g, vb, tid, nthr, (unsigned)pd[kDmItemSlot].cls & 3u); break;
        case 4: dm_fixups<Map>(g, pd, vb, 1, dm_pass_mask<Map>(pd, npos, 1), tid, nthr); break;
        case 5: dm_bulk_stores(mem, map, g, pd, vb, tid, nthr); break;
        default: dm_mirror_stores(mem, map, g, pd, vb, dm_pass_mask<Map>(pd, npos, 2), tid, nthr); break;
    }
}
constexpr int kDmPhases = 7;

constexpr unsigned kDmBlock = 256;          // threads of an engine block
constexpr unsigned kDmIssueThreads = kDmBlock;   // threads that issue the bulk copies

#ifdef __CUDACC__
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

struct DevMemBulk {
    double2* p;
    __device__ __forceinline__ void st(idx_t i, double2 v) const { p[i] = v; }
    __device__ __forceinline__ void bulk_load(double2* sdst, idx_t i, unsigned n, void* bar) const {
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                     ::"r"(smem_u32(sdst)), "l"(p + i), "r"(n * 16u), "r"(smem_u32(bar)) : "memory");
    }
    __device__ __forceinline__ void bulk_store(idx_t i, const double2* ssrc, unsigned n) const {
        asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n"
                     ::"l"(p + i), "r"(smem_u32(ssrc)), "r"(n * 16u) : "memory");
    }
};

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                 " selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

// Error word of the engine: bit 0 set when a wait for staged data ran past its limit.
__device__ unsigned int g_dm_engine_error;

// Bounded wait for the copies of a stage (false: limit reached, error recorded).
__device__ __forceinline__ bool dm_wait_stage(unsigned long long* bar, unsigned parity, unsigned long long limit) {
    for (unsigned long long i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(&g_dm_engine_error, 1u);
    return false;
}

// Per-thread state an op keeps across the items of an engine block: none, except the
// 2-qubit superoperator's tensor-core fragments, built once per block from the kernel
// parameters through the staged block (not in use before the first item).
struct DmNoThreadState {};
template <class Op> struct DmThreadState { using type = DmNoThreadState; };
template <> struct DmThreadState<OpSuper2> { using type = Super2Frag; };

template <class Op>
__device__ __forceinline__ void dm_op_prepare(const Op&, const DmGeom&, DmNoThreadState&, double2*, unsigned,
                                              unsigned) {}
template <class Op>
__device__ __forceinline__ void dm_op_apply(const Op& op, const DmGeom& g, double2* vb, unsigned tid, unsigned nthr,
                                            unsigned iflags, const DmNoThreadState&) {
    op(g, vb, tid, nthr, iflags);
}
__device__ __forceinline__ void dm_op_prepare(const OpSuper2& op, const DmGeom& g, Super2Frag& f, double2* vb,
                                              unsigned tid, unsigned nthr) {
    // the same condition for every block of the launch; only the tensor-core form uses the
    // fragments, and only then is the staged block large enough to stage the entries
    if (!super2_mma_form(g, nthr) || !super2_stage_fits(g)) return;
    for (unsigned i = tid; i < 256; i += nthr) vb[i] = op.s[i];
    __syncthreads();
#pragma unroll
    for (unsigned mt = 0; mt < 4; ++mt)
#pragma unroll
        for (unsigned ks = 0; ks < 8; ++ks) f.a[mt][ks] = super2_afrag(vb, mt, ks, tid & 31u);
    __syncthreads();                                   // read before the first item's copies land
}
__device__ __forceinline__ void dm_op_apply(const OpSuper2& op, const DmGeom& g, double2* vb, unsigned tid,
                                            unsigned nthr, unsigned iflags, const Super2Frag& f) {
    if (super2_mma_form(g, nthr) && super2_stage_fits(g)) op.mma_groups(g, vb, tid, nthr, f);
    else op(g, vb, tid, nthr, iflags);
}

// Blocks per SM the register budget is held to: three blocks with a 64 x 64 staged block
// fill the shared memory, and the bulk copies of one overlap the compute of the others.
// The 2-qubit superoperator keeps 32 tensor-core fragment values per lane across the items
// (64 registers) and gets two.
template <class Op> struct DmMinBlocks { static constexpr int value = 3; };
template <> struct DmMinBlocks<OpSuper2> { static constexpr int value = 2; };

// Persistent engine: block b handles items b, b + G, b + 2G, ...  One item at a time per
// block; with up to three blocks resident per SM (71 KB of shared memory each) the bulk
// copies of one block's item overlap the compute and stores of the others.
template <class Map, class Op>
__global__ void __launch_bounds__(kDmBlock, DmMinBlocks<Op>::value) k_dm_engine(DevMemBulk mem, Map map, DmGeom g, Op op) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_raw);
    DmPos* pd = reinterpret_cast<DmPos*>(smem_raw + 16);
    double2* vb = reinterpret_cast<double2*>(smem_raw + 16 + kDmPosBytes);
    const unsigned tid = threadIdx.x, nthr = blockDim.x;
    const unsigned npos = 1u << (2 * g.h);
    if (blockIdx.x >= g.items) return;
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    typename DmThreadState<Op>::type ts;
    dm_op_prepare(op, g, ts, vb, tid, nthr);
    unsigned parity = 0;
    bool ok = true;
    for (idx_t w = blockIdx.x; w < g.items; w += gridDim.x) {
        dm_setup(map, g, w, pd, tid, nthr);
        __syncthreads();                                   // descriptors ready (and barrier initialised)
        const unsigned iflags = (unsigned)pd[kDmItemSlot].cls;
        if (iflags & 4u) {                                 // nothing in the item changes
            __syncthreads();                               // everyone has read the flags
            continue;
        }
        if (tid == 0) {                                     // arm the barrier with the item's bytes
            unsigned bytes = 0;
            for (unsigned t = 0; t < npos; ++t) bytes += pd[t].bytes;
            mbar_arrive_expect(bar, bytes);
        }
        // every thread issues its share of the bulk loads (a warp issues them one after
        // another, so one issuing warp would cap the block's copy rate)
        fence_proxy_async();
        if (!g.drop_loads) dm_bulk_loads(mem, map, g, pd, vb, bar, tid, nthr);
        const unsigned long long fix0 = dm_pass_mask<Map>(pd, npos, 0);
        const unsigned long long fix1 = dm_pass_mask<Map>(pd, npos, 1);
        const unsigned long long mirr = dm_pass_mask<Map>(pd, npos, 2);
        ok = __syncthreads_and(dm_wait_stage(bar, parity, g.wait_limit) ? 1 : 0) != 0;
        parity ^= 1u;
        if (!ok) break;
        if (fix0) {
            dm_fixups<Map>(g, pd, vb, 0, fix0, tid, nthr);
            __syncthreads();
        }
        dm_op_apply(op, g, vb, tid, nthr, iflags & 3u, ts);
        __syncthreads();
        if (fix1) {
            dm_fixups<Map>(g, pd, vb, 1, fix1, tid, nthr);
            __syncthreads();
        }
        fence_proxy_async();
        __syncthreads();
        dm_bulk_stores(mem, map, g, pd, vb, tid, nthr);
        bulk_commit();
        if (mirr) dm_mirror_stores(mem, map, g, pd, vb, mirr, tid, nthr);
        bulk_wait_read();                                   // the staged block may be refilled
        __syncthreads();
    }
    if (!ok) {
        // give copies still in flight a bounded chance to land before the block exits
        for (unsigned long long i = 0; i < g.wait_limit && !mbar_try_wait(bar, parity); ++i) {
        }
    }
    bulk_wait_all();
}
#endif

}  // namespace orkan
