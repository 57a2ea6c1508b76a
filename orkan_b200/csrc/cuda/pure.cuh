// pure.cuh - statevector kernels: 1-qubit pair streams, 2-qubit quad streams, the
// 3-qubit octet stream of CCX, exp_diag, and the |+> fill.
//
// Arithmetic per gate follows the reference's pair operations in
// src/gate/gate_pure.c:66-268 (zero-multiplication forms for Y/S/Sdg, the sqrt(1/2)
// forms of H/Hy/T/Tdg, host-computed c = cos(theta/2), s = sin(theta/2) for
// Rx/Ry/Rz and c = cos(theta), s = sin(theta) for P), and the quarter/eighth loops of
// cx/cy/cz/swap/ccx (gate_pure.c:282-434).  Gates that change only the |1>-half of a
// pair (Z, S, Sdg, T, Tdg, P) read and write only that half.
//
// Each thread handles kVec independent pairs per loop trip (all loads issued before
// any arithmetic) with a grid-stride loop; consecutive threads take consecutive pair
// indices, so every load and store instruction of a warp is coalesced.
#pragma once

#include "common.cuh"

namespace orkan {

enum PureOp1 : int {
    kOpX = 0, kOpY, kOpZ, kOpH, kOpS, kOpSdg, kOpT, kOpTdg, kOpHy, kOpRx, kOpRy, kOpRz, kOpP,
    kNumOp1
};
enum PureOp2 : int { kOpCX = 0, kOpCY, kOpCZ, kOpSwap, kNumOp2 };

constexpr unsigned kPureThreads = 256;
constexpr unsigned kVec = 4;

#define ORKAN_SQRT1_2 0.70710678118654752440

// c x + s y with one explicitly placed rounding pattern: s y rounded, then one fused
// multiply-add.  Left to the compiler, "c * x + s * y" may be contracted either way, and
// differently in different kernels; written out, every kernel that applies a gate (the
// one-gate kernels, the fused runs, the CPU emulator) gives the same bits.
ORKAN_HD double lin2(double c, double x, double s, double y) {
#ifdef __CUDA_ARCH__
    return __fma_rn(c, x, __dmul_rn(s, y));
#else
    return fma(c, x, s * y);
#endif
}

// Does the op change amplitude a (target bit 0)?
ORKAN_HD constexpr bool op1_touches_a(int op) {
    return !(op == kOpZ || op == kOpS || op == kOpSdg || op == kOpT || op == kOpTdg || op == kOpP);
}

template <int OP>
ORKAN_HD void pair_op(double2& a, double2& b, double c, double s) {
    if (OP == kOpX) {
        const double2 t = a; a = b; b = t;
    } else if (OP == kOpY) {
        const double2 ta = a;
        a = c2(b.y, -b.x);
        b = c2(-ta.y, ta.x);
    } else if (OP == kOpZ) {
        b = c2(-b.x, -b.y);
    } else if (OP == kOpH) {
        const double2 sum = cadd(a, b), dif = csub(a, b);
        a = cscale(sum, ORKAN_SQRT1_2);
        b = cscale(dif, ORKAN_SQRT1_2);
    } else if (OP == kOpHy) {
        const double2 dif = csub(a, b), sum = cadd(a, b);
        a = cscale(dif, ORKAN_SQRT1_2);
        b = cscale(sum, ORKAN_SQRT1_2);
    } else if (OP == kOpS) {
        b = c2(-b.y, b.x);
    } else if (OP == kOpSdg) {
        b = c2(b.y, -b.x);
    } else if (OP == kOpT) {
        b = c2((b.x - b.y) * ORKAN_SQRT1_2, (b.x + b.y) * ORKAN_SQRT1_2);
    } else if (OP == kOpTdg) {
        b = c2((b.x + b.y) * ORKAN_SQRT1_2, (b.y - b.x) * ORKAN_SQRT1_2);
    } else if (OP == kOpP) {
        b = c2(lin2(c, b.x, -s, b.y), lin2(c, b.y, s, b.x));
    } else if (OP == kOpRx) {
        const double2 na = c2(lin2(c, a.x, s, b.y), lin2(c, a.y, -s, b.x));
        const double2 nb = c2(lin2(c, b.x, s, a.y), lin2(c, b.y, -s, a.x));
        a = na; b = nb;
    } else if (OP == kOpRy) {
        const double2 na = c2(lin2(c, a.x, -s, b.x), lin2(c, a.y, -s, b.y));
        const double2 nb = c2(lin2(c, b.x, s, a.x), lin2(c, b.y, s, a.y));
        a = na; b = nb;
    } else if (OP == kOpRz) {
        a = c2(lin2(c, a.x, s, a.y), lin2(c, a.y, -s, a.x));
        b = c2(lin2(c, b.x, -s, b.y), lin2(c, b.y, s, b.x));
    }
}

// One thread's share of a 1-qubit gate on 2^n amplitudes (npairs = 2^(n-1)).
template <int OP, class Mem>
ORKAN_HD void pure1q_thread(const Mem& mem, idx_t npairs, unsigned q, double c, double s,
                            idx_t tid, idx_t nthr) {
    const idx_t stride = idx_t(1) << q;
    for (idx_t k0 = tid; k0 < npairs; k0 += kVec * nthr) {
        idx_t ia[kVec];
        double2 a[kVec], b[kVec];
#pragma unroll
        for (unsigned v = 0; v < kVec; ++v) {
            const idx_t k = k0 + v * nthr;
            ia[v] = insert0(k, q);
            if (k < npairs) {
                if (op1_touches_a(OP)) a[v] = mem.ld(ia[v]);
                b[v] = mem.ld(ia[v] + stride);
            }
        }
#pragma unroll
        for (unsigned v = 0; v < kVec; ++v) {
            if (k0 + v * nthr < npairs) {
                pair_op<OP>(a[v], b[v], c, s);
                if (op1_touches_a(OP)) mem.st(ia[v], a[v]);
                mem.st(ia[v] + stride, b[v]);
            }
        }
    }
}

// 2-qubit gates: quarter loop over indices with both bits zero (nquads = 2^(n-2)).
// qc = control (or q1 for SWAP), qt = target (or q2).
template <int OP, class Mem>
ORKAN_HD void pure2q_thread(const Mem& mem, idx_t nquads, unsigned qc, unsigned qt, idx_t tid, idx_t nthr) {
    const unsigned pos[2] = {qc < qt ? qc : qt, qc < qt ? qt : qc};
    const idx_t bc = idx_t(1) << qc, bt = idx_t(1) << qt;
    for (idx_t k0 = tid; k0 < nquads; k0 += kVec * nthr) {
        idx_t i0[kVec], i1[kVec];
        double2 a[kVec], b[kVec];
#pragma unroll
        for (unsigned v = 0; v < kVec; ++v) {
            const idx_t k = k0 + v * nthr;
            const idx_t base = insert0_sorted(k, pos, 2);
            if (OP == kOpSwap) { i0[v] = base | bc; i1[v] = base | bt; }
            else               { i0[v] = base | bc; i1[v] = base | bc | bt; }
            if (k < nquads) {
                if (OP != kOpCZ) a[v] = mem.ld(i0[v]);
                b[v] = mem.ld(i1[v]);
            }
        }
#pragma unroll
        for (unsigned v = 0; v < kVec; ++v) {
            if (k0 + v * nthr >= nquads) continue;
            if (OP == kOpCZ) {
                mem.st(i1[v], c2(-b[v].x, -b[v].y));
            } else if (OP == kOpCY) {
                mem.st(i0[v], c2(b[v].y, -b[v].x));
                mem.st(i1[v], c2(-a[v].y, a[v].x));
            } else {  // CX, SWAP: exchange
                mem.st(i0[v], b[v]);
                mem.st(i1[v], a[v]);
            }
        }
    }
}

// CCX: eighth loop over indices with all three bits zero (noct = 2^(n-3)).
template <class Mem>
ORKAN_HD void pure_ccx_thread(const Mem& mem, idx_t noct, unsigned c1, unsigned c2q, unsigned t,
                              idx_t tid, idx_t nthr) {
    unsigned pos[3] = {c1, c2q, t};
    for (unsigned a = 0; a < 3; ++a)
        for (unsigned b = a + 1; b < 3; ++b)
            if (pos[b] < pos[a]) { const unsigned tmp = pos[a]; pos[a] = pos[b]; pos[b] = tmp; }
    const idx_t bcc = (idx_t(1) << c1) | (idx_t(1) << c2q), bt = idx_t(1) << t;
    for (idx_t k0 = tid; k0 < noct; k0 += kVec * nthr) {
        idx_t i0[kVec];
        double2 a[kVec], b[kVec];
#pragma unroll
        for (unsigned v = 0; v < kVec; ++v) {
            const idx_t k = k0 + v * nthr;
            i0[v] = insert0_sorted(k, pos, 3) | bcc;
            if (k < noct) { a[v] = mem.ld(i0[v]); b[v] = mem.ld(i0[v] | bt); }
        }
#pragma unroll
        for (unsigned v = 0; v < kVec; ++v) {
            if (k0 + v * nthr >= noct) continue;
            mem.st(i0[v], b[v]);
            mem.st(i0[v] | bt, a[v]);
        }
    }
}

// exp_diag on a statevector: psi_x *= exp(-i diag[x] t)  (reference src/circ/circ_pure.c:21-33).
template <class Mem, class MemR>
ORKAN_HD void pure_exp_diag_thread(const Mem& mem, const MemR& diag, idx_t dim, double t, idx_t tid, idx_t nthr) {
    for (idx_t x0 = tid; x0 < dim; x0 += kVec * nthr) {
        double2 v[kVec];
        double ang[kVec];
#pragma unroll
        for (unsigned u = 0; u < kVec; ++u) {
            const idx_t x = x0 + u * nthr;
            if (x < dim) { v[u] = mem.ld(x); ang[u] = diag.ld(x) * t; }
        }
#pragma unroll
        for (unsigned u = 0; u < kVec; ++u) {
            const idx_t x = x0 + u * nthr;
            if (x >= dim) continue;
            double sn, cs;
            sincos(ang[u], &sn, &cs);
            mem.st(x, c2(cs * v[u].x + sn * v[u].y, cs * v[u].y - sn * v[u].x));
        }
    }
}

// Fill stored elements with a value.  For the tiled layout with dim < tile side only the
// dim x dim corner of the single tile is written (reference state_tiled.c:100-113).
template <class Mem>
ORKAN_HD void fill_thread(const Mem& mem, idx_t len, double2 val, unsigned corner_log_tile, idx_t corner_dim,
                          idx_t tid, idx_t nthr) {
    for (idx_t i = tid; i < len; i += nthr) {
        if (corner_dim) {
            const idx_t lr = i >> corner_log_tile, lc = i & ((idx_t(1) << corner_log_tile) - 1);
            if (lr >= corner_dim || lc >= corner_dim) continue;
        }
        mem.st(i, val);
    }
}

#ifdef __CUDACC__
template <int OP>
__global__ void __launch_bounds__(kPureThreads) k_pure1q(DevMem mem, idx_t npairs, unsigned q, double c, double s) {
    pure1q_thread<OP>(mem, npairs, q, c, s, (idx_t)blockIdx.x * blockDim.x + threadIdx.x,
                      (idx_t)gridDim.x * blockDim.x);
}
template <int OP>
__global__ void __launch_bounds__(kPureThreads) k_pure2q(DevMem mem, idx_t nquads, unsigned qc, unsigned qt) {
    pure2q_thread<OP>(mem, nquads, qc, qt, (idx_t)blockIdx.x * blockDim.x + threadIdx.x,
                      (idx_t)gridDim.x * blockDim.x);
}
static __global__ void __launch_bounds__(kPureThreads) k_pure_ccx(DevMem mem, idx_t noct, unsigned c1, unsigned c2q, unsigned t) {
    pure_ccx_thread(mem, noct, c1, c2q, t, (idx_t)blockIdx.x * blockDim.x + threadIdx.x,
                    (idx_t)gridDim.x * blockDim.x);
}
static __global__ void __launch_bounds__(kPureThreads) k_pure_exp_diag(DevMem mem, DevMemR diag, idx_t dim, double t) {
    pure_exp_diag_thread(mem, diag, dim, t, (idx_t)blockIdx.x * blockDim.x + threadIdx.x,
                         (idx_t)gridDim.x * blockDim.x);
}
static __global__ void __launch_bounds__(kPureThreads) k_fill(DevMem mem, idx_t len, double2 val, unsigned clt, idx_t cdim) {
    fill_thread(mem, len, val, clt, cdim, (idx_t)blockIdx.x * blockDim.x + threadIdx.x,
                (idx_t)gridDim.x * blockDim.x);
}
#endif

}  // namespace orkan
