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

inline PhaseGeom phase_geometry(unsigned n, unsigned ls_max) {
    PhaseGeom g;
    g.d = idx_t(1) << n;
    g.ls = ls_max < n ? ls_max : n;
    g.nseg = g.d >> g.ls;
    g.items = g.nseg * (g.nseg + 1) / 2;
    return g;
}

// Phase of a k-qubit diagonal gate: phi(x) = phase[local(x)], local(x) = sum_j bit(x, q[j]) << (k-1-j).
struct GateFactor {
    unsigned k;
    unsigned q[3];
    double2 phase[8];
    ORKAN_HD unsigned local(idx_t x) const {
        unsigned l = 0;
        for (unsigned j = 0; j < k; ++j) l = (l << 1) | (unsigned)((x >> q[j]) & 1u);
        return l;
    }
    // returns false when the factor is exactly one (element unchanged)
    ORKAN_HD bool factor(idx_t r, idx_t c, double2* f) const {
        const unsigned lr = local(r), lc = local(c);
        if (lr == lc) return false;
        *f = cmulc(phase[lr], phase[lc]);
        return !(f->x == 1.0 && f->y == 0.0);
    }
};

// exp_diag: tab[x] = (cos(diag[x] t), sin(diag[x] t)); factor e^{-i(d_r - d_c)t} formed as in
// the reference: f_re = cr*cc + sr*sc, f_im = -sr*cc + cr*sc.
template <class MemR2>
struct TableFactor {
    MemR2 tab;
    ORKAN_HD bool factor(idx_t r, idx_t c, double2* f) const {
        const double2 pr = tab.ld(r), pc = tab.ld(c);
        f->x = pr.x * pc.x + pr.y * pc.y;
        f->y = -pr.y * pc.x + pr.x * pc.y;
        return true;
    }
};

// Apply rho' = f * rho  (complex product written out as the reference does:
// re' = f_re*re - f_im*im, im' = f_re*im + f_im*re).
ORKAN_HD double2 phase_apply(double2 f, double2 v) {
    return c2(f.x * v.x - f.y * v.y, f.x * v.y + f.y * v.x);
}

constexpr unsigned kPhaseEpt = 4;   // elements per thread per trip: loads issued together

template <class Map, class Mem, class Factor>
ORKAN_HD void dm_phase_item(const Mem& mem, const Map& map, const PhaseGeom& g, const Factor& fac,
                            idx_t w, unsigned tid, unsigned nthr) {
    idx_t u, v;
    tri_unrank(w, &u, &v);
    const unsigned ls = g.ls, S = 1u << ls;
    const idx_t R = u << ls, C = v << ls;
    const unsigned total = S * S;
    const bool diag = (u == v);
    const bool mirror = Map::kMirrors && !diag && map.same_storage_block(R, C);
    for (unsigned e0 = tid; e0 < total; e0 += nthr * kPhaseEpt) {
        idx_t addr[kPhaseEpt], maddr[kPhaseEpt];
        double2 f[kPhaseEpt], val[kPhaseEpt];
        bool act[kPhaseEpt];
#pragma unroll
        for (unsigned k = 0; k < kPhaseEpt; ++k) {
            const unsigned e = e0 + k * nthr;
            act[k] = false;
            if (e >= total) continue;
            const unsigned line = e >> ls, pos = e & (S - 1);
            unsigned i, j;
            if (Map::kRowContig) { i = pos; j = line; } else { i = line; j = pos; }
            if (diag && i <= j) continue;
            if (!fac.factor(R + i, C + j, &f[k])) continue;
            act[k] = true;
            addr[k] = map.at(R + i, C + j);
            maddr[k] = (Map::kMirrors && (diag || mirror)) ? map.at(C + j, R + i) : addr[k];
            val[k] = mem.ld(addr[k]);
        }
#pragma unroll
        for (unsigned k = 0; k < kPhaseEpt; ++k) {
            if (!act[k]) continue;
            const double2 nv = phase_apply(f[k], val[k]);
            mem.st(addr[k], nv);
            if (maddr[k] != addr[k]) mem.st(maddr[k], cconj(nv));
        }
    }
}

#ifdef __CUDACC__
template <class Map, class Factor>
__global__ void __launch_bounds__(kPhaseThreads) k_dm_phase(DevMem mem, Map map, PhaseGeom g, Factor fac) {
    for (idx_t w = blockIdx.x; w < g.items; w += gridDim.x)
        dm_phase_item(mem, map, g, fac, w, threadIdx.x, blockDim.x);
}
#endif

}  // namespace orkan
