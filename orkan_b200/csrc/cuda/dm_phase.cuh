// dm_phase.cuh - elementwise phase updates of a density matrix:
//     rho_rc *= phi(r) * conj(phi(c))
// for diagonal gates (Z, S, Sdg, T, Tdg, P, Rz, CZ; reference p_packed at
// src/gate/packed/gate_packed_1q.c:481-523, gate_tiled_rz.c, gate_packed_cz.c:23-80)
// and for exp_diag (reference src/circ/circ_packed.c:28-71, circ_tiled.c:25-105, which
// precompute cos/sin per index and form the pair phase with the product identity).
//
// Work is cut into S x S sub-tiles of the lower triangle.  Diagonal elements are never
// touched (their factor is |phi|^2 = 1).  Elements whose factor is exactly 1 are neither
// read nor written, so a Z gate moves only the sectors it changes.  On the tiled layout
// the upper half of diagonal tiles is rewritten as the conjugate of the updated lower
// half (as circ_tiled.c does), never computed independently.
#pragma once

#include "common.cuh"

namespace orkan {

constexpr unsigned kPhaseThreads = 128;

struct PhaseGeom {
    idx_t d;
    unsigned ls;        // log2 of sub-tile side
    idx_t nseg;         // d >> ls
    idx_t items;        // nseg * (nseg + 1) / 2
};

// The sub-tile side is at most kPhaseMaxS (ls_max is clamped to 5).
inline PhaseGeom phase_geometry(unsigned n, unsigned ls_max) {
    if (ls_max > 5) ls_max = 5;
    PhaseGeom g;
    g.d = idx_t(1) << n;
    g.ls = ls_max < n ? ls_max : n;
    g.nseg = g.d >> g.ls;
    g.items = g.nseg * (g.nseg + 1) / 2;
    return g;
}

// Factor forms.  factor(r, c, &f) returns false when the element is unchanged.
//
// 1-qubit diagonal gate diag(1, ph1) on qubit q: f = ph1 when bit q of r is set and of c
// clear, conj(ph1) in the opposite case, unchanged otherwise.
struct GateFactor1 {
    unsigned q;
    double2 ph1;
    // can any element of the S x S item at (R, C) change?  (bit q is constant over the item
    // when q >= log2 S)
    ORKAN_HD bool item_active(idx_t R, idx_t C, unsigned ls) const {
        return q < ls || (((R ^ C) >> q) & 1u);
    }
    ORKAN_HD bool factor(idx_t r, idx_t c, double2* f) const {
        const unsigned br = (unsigned)(r >> q) & 1u, bc = (unsigned)(c >> q) & 1u;
        if (br == bc) return false;
        *f = br ? ph1 : cconj(ph1);
        return true;
    }
};

// Controlled phase (CZ and every diagonal gate whose phases are 1 except on the all-ones
// local index): phi(x) = ph when every bit of mask is set in x, else 1.  The element changes
// when exactly one of r, c has them all: f = ph for r, conj(ph) for c.
struct GateFactorCtrl {
    unsigned long long mask;
    double2 ph;
    // the mask bits at or above log2 S are constant over the item: rows (columns) can meet
    // the mask only when R (C) has all of them
    ORKAN_HD bool item_active(idx_t R, idx_t C, unsigned ls) const {
        const unsigned long long hi = mask & ~((1ull << ls) - 1ull);
        return (((unsigned long long)R & hi) == hi) || (((unsigned long long)C & hi) == hi);
    }
    ORKAN_HD bool factor(idx_t r, idx_t c, double2* f) const {
        const bool br = ((unsigned long long)r & mask) == mask, bc = ((unsigned long long)c & mask) == mask;
        if (br == bc) return false;
        *f = br ? ph : cconj(ph);
        return true;
    }
};

// k-qubit diagonal gate (k <= 3): phi(x) = phase[local(x)], local(x) = sum_j bit(x, q[j]) << (k-1-j);
// f = phi(r) conj(phi(c)); equal local indices give |phi|^2 = 1 and are skipped.
struct GateFactor {
    unsigned k;
    unsigned q[3];
    double2 phase[8];
    ORKAN_HD bool item_active(idx_t, idx_t, unsigned) const { return true; }
    ORKAN_HD unsigned local(idx_t x) const {
        unsigned l = 0;
        for (unsigned j = 0; j < k; ++j) l = (l << 1) | (unsigned)((x >> q[j]) & 1u);
        return l;
    }
    ORKAN_HD bool factor(idx_t r, idx_t c, double2* f) const {
        const unsigned lr = local(r), lc = local(c);
        if (lr == lc) return false;
        double2 pr = phase[0], pc = phase[0];
        for (unsigned l = 1; l < 8; ++l) {      // select without dynamic indexing
            if (l == lr) pr = phase[l];
            if (l == lc) pc = phase[l];
        }
        *f = cmulc(pr, pc);
        return !(f->x == 1.0 && f->y == 0.0);
    }
};

// exp_diag: tab[x] = (cos(diag[x] t), sin(diag[x] t)); the factor e^{-i(d_r - d_c)t} is
// formed as in the reference: f_re = cr*cc + sr*sc, f_im = -sr*cc + cr*sc.  The S row and S
// column entries an item needs are staged in shared memory once per item (kStaged), so the
// element loop reads the state and two shared-memory entries instead of the table.
template <class MemR2>
struct TableFactor {
    MemR2 tab;
    static constexpr bool kStaged = true;
    ORKAN_HD bool item_active(idx_t, idx_t, unsigned) const { return true; }
    ORKAN_HD static void combine(double2 pr, double2 pc, double2* f) {
        f->x = pr.x * pc.x + pr.y * pc.y;
        f->y = -pr.y * pc.x + pr.x * pc.y;
    }
    ORKAN_HD bool factor(idx_t r, idx_t c, double2* f) const {
        combine(tab.ld(r), tab.ld(c), f);
        return true;
    }
    // srow[i] = tab[R + i], scol[j] = tab[C + j] for i, j < S
    ORKAN_HD void stage(idx_t R, idx_t C, unsigned S, double2* srow, double2* scol, unsigned tid,
                        unsigned nthr) const {
        for (unsigned i = tid; i < 2 * S; i += nthr) {
            if (i < S) srow[i] = tab.ld(R + i);
            else scol[i - S] = tab.ld(C + i - S);
        }
    }
};

// Factors without staged entries.
template <class F>
struct PhaseStaged { static constexpr bool value = false; };
template <class M>
struct PhaseStaged<TableFactor<M>> { static constexpr bool value = true; };

// Apply rho' = f * rho  (complex product written out as the reference does:
// re' = f_re*re - f_im*im, im' = f_re*im + f_im*re).
ORKAN_HD double2 phase_apply(double2 f, double2 v) {
    return c2(f.x * v.x - f.y * v.y, f.x * v.y + f.y * v.x);
}

constexpr unsigned kPhaseEpt = 4;     // elements per thread per trip: loads issued together

// Row u, column v of the lower-triangular item index w = u(u+1)/2 + v (single-precision
// estimate, corrected exactly in integers).
ORKAN_HD void tri_unrank_fast(idx_t w, idx_t* u, idx_t* v) {
    idx_t uu = (idx_t)((sqrtf(8.0f * (float)w + 1.0f) - 1.0f) * 0.5f);
    while (uu > 0 && uu * (uu + 1) / 2 > w) --uu;
    while ((uu + 1) * (uu + 2) / 2 <= w) ++uu;
    *u = uu;
    *v = w - uu * (uu + 1) / 2;
}

// Staging phase of item w for staged factors (all threads; a barrier follows).
template <class Factor>
ORKAN_HD void dm_phase_stage(const PhaseGeom& g, const Factor& fac, idx_t w, double2* srow, double2* scol,
                             unsigned tid, unsigned nthr) {
    if constexpr (PhaseStaged<Factor>::value) {
        idx_t u, v;
        tri_unrank_fast(w, &u, &v);
        fac.stage(u << g.ls, v << g.ls, 1u << g.ls, srow, scol, tid, nthr);
    } else {
        (void)g; (void)fac; (void)w; (void)srow; (void)scol; (void)tid; (void)nthr;
    }
}

template <class Map, class Mem, class Factor>
ORKAN_HD void dm_phase_item(const Mem& mem, const Map& map, const PhaseGeom& g, const Factor& fac,
                            idx_t w, unsigned tid, unsigned nthr, const double2* srow = nullptr,
                            const double2* scol = nullptr) {
    idx_t u, v;
    tri_unrank_fast(w, &u, &v);
    const unsigned ls = g.ls, S = 1u << ls;
    const idx_t R = u << ls, C = v << ls;
    if (!fac.item_active(R, C, ls)) return;
    const unsigned total = S * S;
    const bool diag = (u == v);
    const idx_t base = map.at(R, C);
    const idx_t gcol = Map::kRowContig ? map.d - C - 1 : 0;
    const unsigned lt = map.log_tdim();
    // tiled: an item inside a diagonal tile has its mirror image stored too
    const bool mir = Map::kMirrors && (diag || map.same_storage_block(R, C));
    const idx_t mbase = diag ? base : (mir ? map.at(C, R) : 0);
    for (unsigned e0 = tid; e0 < total; e0 += nthr * kPhaseEpt) {
        idx_t addr[kPhaseEpt];
        double2 val[kPhaseEpt], f[kPhaseEpt];
        unsigned ij[kPhaseEpt];
        bool act[kPhaseEpt];
#pragma unroll
        for (unsigned k = 0; k < kPhaseEpt; ++k) {
            const unsigned e = e0 + k * nthr;
            act[k] = false;
            if (e >= total) continue;
            const unsigned line = e >> ls, p = e & (S - 1);
            unsigned i, j;
            if (Map::kRowContig) { i = p; j = line; } else { i = line; j = p; }
            if (diag && i <= j) continue;
            if constexpr (PhaseStaged<Factor>::value) Factor::combine(srow[i], scol[j], &f[k]);
            else if (!fac.factor(R + i, C + j, &f[k])) continue;
            act[k] = true;
            ij[k] = (i << 16) | j;
            addr[k] = Map::kRowContig ? base + (idx_t)line * gcol - (idx_t)((line * (line - 1)) >> 1) + p
                                      : base + ((idx_t)line << lt) + p;
            val[k] = mem.ld(addr[k]);
        }
#pragma unroll
        for (unsigned k = 0; k < kPhaseEpt; ++k) {
            if (!act[k]) continue;
            const double2 nv = phase_apply(f[k], val[k]);
            mem.st(addr[k], nv);
            if (Map::kMirrors && mir) mem.st(mbase + ((idx_t)(ij[k] & 0xffffu) << lt) + (ij[k] >> 16), cconj(nv));
        }
    }
}

#ifdef __CUDACC__
template <class Map, class Factor>
__global__ void __launch_bounds__(kPhaseThreads) k_dm_phase(DevMem mem, Map map, PhaseGeom g, Factor fac) {
    __shared__ double2 srow[32], scol[32];
    for (idx_t w = blockIdx.x; w < g.items; w += gridDim.x) {
        if constexpr (PhaseStaged<Factor>::value) {
            __syncthreads();                         // the previous item's entries are read
            dm_phase_stage(g, fac, w, srow, scol, threadIdx.x, blockDim.x);
            __syncthreads();
        }
        dm_phase_item(mem, map, g, fac, w, threadIdx.x, blockDim.x, srow, scol);
    }
}
#endif

}  // namespace orkan
