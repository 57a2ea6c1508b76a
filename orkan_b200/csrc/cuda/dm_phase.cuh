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

constexpr unsigned kPhaseThreads = 256;

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

// Phase of a k-qubit diagonal gate: phi(x) = phase[local(x)], local(x) = sum_j bit(x, q[j]) << (k-1-j).
// The element factor is phi(r) conj(phi(c)); rows and columns with the same local index
// get factor |phi|^2 = 1 and are skipped.
struct GateFactor {
    unsigned k;
    unsigned q[3];
    double2 phase[8];
    static constexpr bool kKeyed = true;
    ORKAN_HD unsigned key(idx_t x) const {
        unsigned l = 0;
        for (unsigned j = 0; j < k; ++j) l = (l << 1) | (unsigned)((x >> q[j]) & 1u);
        return l;
    }
    ORKAN_HD double2 value(idx_t x) const { return phase[key(x)]; }
    ORKAN_HD double2 combine(double2 rv, double2 cv) const { return cmulc(rv, cv); }
};

// exp_diag: tab[x] = (cos(diag[x] t), sin(diag[x] t)); the factor e^{-i(d_r - d_c)t} is
// formed as in the reference: f_re = cr*cc + sr*sc, f_im = -sr*cc + cr*sc.
template <class MemR2>
struct TableFactor {
    MemR2 tab;
    static constexpr bool kKeyed = false;
    ORKAN_HD unsigned key(idx_t) const { return 0; }
    ORKAN_HD double2 value(idx_t x) const { return tab.ld(x); }
    ORKAN_HD double2 combine(double2 rv, double2 cv) const { return cmulc(cv, rv); }
};

// Apply rho' = f * rho  (complex product written out as the reference does:
// re' = f_re*re - f_im*im, im' = f_re*im + f_im*re).
ORKAN_HD double2 phase_apply(double2 f, double2 v) {
    return c2(f.x * v.x - f.y * v.y, f.x * v.y + f.y * v.x);
}

constexpr unsigned kPhaseMaxS = 32;   // sub-tile side of the phase pass
constexpr unsigned kPhaseEpt = 4;     // elements per thread per trip: loads issued together

// Per-item staging in shared memory: factor values and skip keys of the S rows and S columns.
struct PhaseShared {
    double2 rv[kPhaseMaxS], cv[kPhaseMaxS];
    unsigned char rk[kPhaseMaxS], ck[kPhaseMaxS];
};

template <class Factor>
ORKAN_HD void dm_phase_setup(const PhaseGeom& g, const Factor& fac, idx_t w, PhaseShared* sh, unsigned tid,
                             unsigned nthr) {
    idx_t u, v;
    tri_unrank(w, &u, &v);
    const unsigned S = 1u << g.ls;
    for (unsigned t = tid; t < 2 * S; t += nthr) {
        if (t < S) {
            const idx_t r = (u << g.ls) + t;
            sh->rv[t] = fac.value(r);
            sh->rk[t] = (unsigned char)fac.key(r);
        } else {
            const idx_t c = (v << g.ls) + (t - S);
            sh->cv[t - S] = fac.value(c);
            sh->ck[t - S] = (unsigned char)fac.key(c);
        }
    }
}

template <class Map, class Mem, class Factor>
ORKAN_HD void dm_phase_item(const Mem& mem, const Map& map, const PhaseGeom& g, const Factor& fac,
                            const PhaseShared* sh, idx_t w, unsigned tid, unsigned nthr) {
    idx_t u, v;
    tri_unrank(w, &u, &v);
    const unsigned ls = g.ls, S = 1u << ls;
    const idx_t R = u << ls, C = v << ls;
    const unsigned total = S * S;
    const bool diag = (u == v);
    const idx_t base = map.at(R, C);
    const idx_t gcol = Map::kRowContig ? map.d - C - 1 : 0;
    const unsigned lt = map.log_tdim();
    // tiled: the item lies in a diagonal tile, so its mirror image is stored too
    const bool mir = Map::kMirrors && (diag || map.same_storage_block(R, C));
    const idx_t mbase = diag ? base : (mir ? map.at(C, R) : 0);
    for (unsigned e0 = tid; e0 < total; e0 += nthr * kPhaseEpt) {
        idx_t addr[kPhaseEpt];
        double2 val[kPhaseEpt];
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
            if (Factor::kKeyed && sh->rk[i] == sh->ck[j]) continue;
            act[k] = true;
            ij[k] = (i << 8) | j;
            addr[k] = Map::kRowContig ? base + (idx_t)line * gcol - (idx_t)((line * (line - 1)) >> 1) + p
                                      : base + ((idx_t)line << lt) + p;
            val[k] = mem.ld(addr[k]);
        }
#pragma unroll
        for (unsigned k = 0; k < kPhaseEpt; ++k) {
            if (!act[k]) continue;
            const unsigned i = ij[k] >> 8, j = ij[k] & 0xffu;
            const double2 nv = phase_apply(fac.combine(sh->rv[i], sh->cv[j]), val[k]);
            mem.st(addr[k], nv);
            if (Map::kMirrors && mir) mem.st(mbase + ((idx_t)j << lt) + i, cconj(nv));
        }
    }
}

#ifdef __CUDACC__
template <class Map, class Factor>
__global__ void __launch_bounds__(kPhaseThreads) k_dm_phase(DevMem mem, Map map, PhaseGeom g, Factor fac) {
    __shared__ PhaseShared sh;
    for (idx_t w = blockIdx.x; w < g.items; w += gridDim.x) {
        dm_phase_setup(g, fac, w, &sh, threadIdx.x, blockDim.x);
        __syncthreads();
        dm_phase_item(mem, map, g, fac, &sh, w, threadIdx.x, blockDim.x);
        __syncthreads();
    }
}
#endif

}  // namespace orkan
