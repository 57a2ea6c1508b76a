// common.cuh - complex arithmetic, bit helpers and storage maps shared by every kernel.
//
// Everything here is __host__ __device__ so that the kernels' index logic can also
// run in the CPU emulator used by the test suite (tests/emu), which bounds-checks
// every access the kernels make.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#define ORKAN_HD __host__ __device__ __forceinline__

namespace orkan {

typedef uint64_t idx_t;

// ---------------------------------------------------------------------------------
// complex128 as double2 {x = re, y = im}; 16 bytes, same layout as C99 double _Complex
// ---------------------------------------------------------------------------------
ORKAN_HD double2 c2(double re, double im) { double2 r; r.x = re; r.y = im; return r; }
ORKAN_HD double2 cadd(double2 a, double2 b) { return c2(a.x + b.x, a.y + b.y); }
ORKAN_HD double2 csub(double2 a, double2 b) { return c2(a.x - b.x, a.y - b.y); }
ORKAN_HD double2 cmul(double2 a, double2 b) { return c2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
ORKAN_HD double2 cconj(double2 a) { return c2(a.x, -a.y); }
ORKAN_HD double2 cscale(double2 a, double s) { return c2(a.x * s, a.y * s); }
// a * conj(b)
ORKAN_HD double2 cmulc(double2 a, double2 b) { return c2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }

// ---------------------------------------------------------------------------------
// bit helpers (the reference's insertBit0 / insertBits2_0, src/internal/index.h:28-44)
// ---------------------------------------------------------------------------------
// Insert a zero bit at position pos of v.
ORKAN_HD idx_t insert0(idx_t v, unsigned pos) {
    const idx_t lo = v & ((idx_t(1) << pos) - 1);
    return lo | ((v - lo) << 1);
}
// Insert zero bits at the ascending positions p[0] < p[1] < ... < p[k-1].
ORKAN_HD idx_t insert0_sorted(idx_t v, const unsigned* p, unsigned k) {
    for (unsigned j = 0; j < k; ++j) v = insert0(v, p[j]);
    return v;
}
// Scatter the low bits of a onto the positions p[0..k-1] (bit j of a -> bit p[j]).
ORKAN_HD idx_t spread_bits(unsigned a, const unsigned* p, unsigned k) {
    idx_t r = 0;
    for (unsigned j = 0; j < k; ++j) r |= idx_t((a >> j) & 1u) << p[j];
    return r;
}

// Index of the lowest set bit of a non-zero 64-bit word.
ORKAN_HD unsigned ctz64(unsigned long long x) {
#ifdef __CUDA_ARCH__
    return (unsigned)(__ffsll((long long)x) - 1);
#else
    return (unsigned)__builtin_ctzll(x);
#endif
}

ORKAN_HD unsigned popc64(unsigned long long x) {
#ifdef __CUDA_ARCH__
    return (unsigned)__popcll(x);
#else
    return (unsigned)__builtin_popcountll(x);
#endif
}

// Row u, column v of the lower-triangular item index w = u(u+1)/2 + v: single-precision
// estimate corrected exactly in integers.
ORKAN_HD void tri_unrank_f(idx_t w, idx_t* u, idx_t* v) {
    idx_t uu = (idx_t)((sqrtf(8.0f * (float)w + 1.0f) - 1.0f) * 0.5f);
    while (uu > 0 && uu * (uu + 1) / 2 > w) --uu;
    while ((uu + 1) * (uu + 2) / 2 <= w) ++uu;
    *u = uu;
    *v = w - uu * (uu + 1) / 2;
}

// Row r of the lower-triangular enumeration w = u*(u+1)/2 + v, v <= u.
ORKAN_HD void tri_unrank(idx_t w, idx_t* u, idx_t* v) {
    idx_t uu = (idx_t)((sqrt(8.0 * (double)w + 1.0) - 1.0) * 0.5);
    while (uu * (uu + 1) / 2 > w) --uu;
    while ((uu + 1) * (uu + 2) / 2 <= w) ++uu;
    *u = uu;
    *v = w - uu * (uu + 1) / 2;
}

// ---------------------------------------------------------------------------------
// Storage maps.  at(r, c) is the storage index of density-matrix element (r, c).
// ---------------------------------------------------------------------------------
// MIXED_PACKED: lower triangle column-major (reference src/internal/index.h:57-68).
// Valid for r >= c.  Contiguous along r inside a column.
struct PackedMap {
    idx_t d;
    ORKAN_HD idx_t col_start(idx_t c) const { return c * (2 * d - c + 1) / 2; }
    ORKAN_HD idx_t at(idx_t r, idx_t c) const { return col_start(c) + (r - c); }
    ORKAN_HD idx_t len() const { return (d / 2) * (d + 1) + (d == 1 ? 1 : 0); }
    static constexpr bool kRowContig = true;   // consecutive rows are adjacent
    static constexpr bool kMirrors = false;    // no stored upper-triangle copies
    ORKAN_HD bool same_storage_block(idx_t, idx_t) const { return false; }
    ORKAN_HD unsigned log_tdim() const { return 0; }
};

// MIXED_TILED: lower-triangular grid of 2^L x 2^L tiles, tiles in row-major tile
// order, elements row-major inside a tile (reference src/internal/index.h:79-88).
// Valid for (r >> L) >= (c >> L); diagonal tiles hold both triangles.
struct TiledMap {
    idx_t d;
    unsigned L;
    ORKAN_HD idx_t tdim() const { return idx_t(1) << L; }
    ORKAN_HD idx_t at(idx_t r, idx_t c) const {
        const idx_t tr = r >> L, tc = c >> L, m = tdim() - 1;
        return ((tr * (tr + 1) / 2 + tc) << (2 * L)) + ((r & m) << L) + (c & m);
    }
    ORKAN_HD idx_t len() const {
        const idx_t nt = (d + tdim() - 1) >> L;
        return (nt * (nt + 1) / 2) << (2 * L);
    }
    static constexpr bool kRowContig = false;  // consecutive columns are adjacent
    static constexpr bool kMirrors = true;     // diagonal tiles store the upper half too
    // Do rows r and c fall into the same tile row (so (r,c) and (c,r) share a tile)?
    ORKAN_HD bool same_storage_block(idx_t r, idx_t c) const { return (r >> L) == (c >> L); }
    ORKAN_HD unsigned log_tdim() const { return L; }
};

// ---------------------------------------------------------------------------------
// Memory accessor.  On the GPU a raw pointer; the CPU emulator substitutes a
// checking accessor with the same interface.
// ---------------------------------------------------------------------------------
#ifdef __CUDACC__
struct DevMem {
    double2* p;
    __device__ __forceinline__ double2 ld(idx_t i) const { return p[i]; }
    __device__ __forceinline__ void st(idx_t i, double2 v) const { p[i] = v; }
};
struct DevMemR {   // read-only real array
    const double* p;
    __device__ __forceinline__ double ld(idx_t i) const { return __ldg(p + i); }
};
#endif

}  // namespace orkan
