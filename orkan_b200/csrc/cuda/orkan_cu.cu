// orkan_cu.cu - the C-ABI launch layer (include/orkan_cu.h): argument checks, launch
// geometry, template dispatch, and the per-device scratch buffer used by reductions
// and by the exp_diag phase tables.
#include "common.cuh"
#include "dm_engine.cuh"
#include "dm_phase.cuh"
#include "launch.cuh"
#include "pure.cuh"
#include "pure_fused.cuh"
#include "reduce.cuh"
#include "scratch.cuh"

#include "../../../include/orkan_cu.h"

#include <atomic>
#include <chrono>
#include <cstring>
#include <stdlib.h>
#include <mutex>

using namespace orkan;

namespace {
std::atomic<unsigned long long> g_launches{0};
std::atomic<int> g_sm_count[64];
}  // namespace

namespace orkan {

int sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    int v = g_sm_count[dev].load(std::memory_order_relaxed);
    if (v <= 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        g_sm_count[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

int finish_launch() {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    return (int)cudaGetLastError();
}

// Two items per block by default (measured at 14 q with 4 elements per thread per trip: T on
// every target 3754 against 3393 GB/s tiled, 2503 against 2545 packed, exp_diag unchanged).
unsigned phase_items_per_block() {
    static const unsigned v = [] {
        const char* e = getenv("ORKAN_PHASE_ITEMS");
        const int x = e ? atoi(e) : 2;
        return (x == 1 || x == 2 || x == 4 || x == 8) ? (unsigned)x : 2u;
    }();
    return v;
}

}  // namespace orkan

namespace {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Test hook of the engine's bounded waits (orkan_cu_engine_test_wait): 0 polls = the default.
std::atomic<unsigned long long> g_engine_test_polls{0};
std::atomic<unsigned> g_engine_test_drop{0};

inline double2 ld_c(const double* p, unsigned i) { return c2(p[2 * i], p[2 * i + 1]); }

// ---- density-matrix engine dispatch -------------------------------------------------
template <class Kern>
unsigned engine_grid(Kern kern, size_t smem, idx_t items) {
    static bool attr = false;
    if (!attr) {
        // the dynamic limit leaves room for the kernel's static shared memory (the 2-qubit
        // superoperator stages its entries there): static + dynamic may not exceed 227 KB
        cudaFuncAttributes fa;
        size_t stat = 0;
        if (cudaFuncGetAttributes(&fa, kern) == cudaSuccess) stat = fa.sharedSizeBytes;
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(227 * 1024 - stat));
        attr = true;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kDmBlock, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return grid_for(1, items, (unsigned)(sm_count() * per_sm));
}

template <class Op>
int launch_engine_map(int layout, unsigned log_tile, void* rho, unsigned n, DmGeom g, Op op, cudaStream_t st) {
    const size_t smem = dm_block_smem_bytes(g);
    if (const unsigned long long polls = g_engine_test_polls.load(std::memory_order_relaxed)) {
        g.wait_limit = polls;
        g.drop_loads = g_engine_test_drop.load(std::memory_order_relaxed);
    }
    dm_orient(op, layout == 1);               // the packed layout stages rho^T
    DevMemBulk mem{static_cast<double2*>(rho)};
    if (layout == 1) {
        auto kern = k_dm_engine<PackedMap, Op>;
        const unsigned grid = engine_grid(kern, smem, g.items);
        kern<<<grid, kDmBlock, smem, st>>>(mem, PackedMap{idx_t(1) << n}, g, op);
    } else {
        auto kern = k_dm_engine<TiledMap, Op>;
        const unsigned grid = engine_grid(kern, smem, g.items);
        kern<<<grid, kDmBlock, smem, st>>>(mem, TiledMap{idx_t(1) << n, log_tile}, g, op);
    }
    return finish_launch();
}

// Largest engine block side when at most one gate qubit lies above the sub-tile (a power of
// two in [8, 64]).  Tuning knob: environment variable ORKAN_DM_MAX_V, read once.
unsigned dm_max_v_low() {
    static unsigned v = 0;
    if (!v) {
        unsigned x = 64;
        if (const char* e = getenv("ORKAN_DM_MAX_V")) {
            const unsigned y = (unsigned)atoi(e);
            if (y == 8 || y == 16 || y == 32 || y == 64) x = y;
        }
        v = x;
    }
    return v;
}

inline bool layout_ok(int layout, unsigned log_tile) {
    if (layout == 1) return true;
    if (layout == 2) return log_tile >= 1 && log_tile <= 8;
    return false;
}

// sub-tile side limit: tiles for the tiled layout, 64 for packed
inline unsigned ls_max_for(int layout, unsigned log_tile) { return layout == 2 ? log_tile : 6u; }

// Result slots of mean / matel_diag in mapped pinned host memory (per device, allocated
// on first use): the folding block writes the results there, then a sequence number, so the
// host reads the value as soon as the number appears, without a device-to-host copy and
// without waiting for the stream to drain.
struct MappedOut {
    double* host = nullptr;
    double* dev = nullptr;
    double seq = 0.0;          // last sequence number issued on this device
};
std::mutex g_mapped_mu;
MappedOut g_mapped[64];

// The device's slots and the next sequence number.
int mapped_out(MappedOut* m) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    if (dev < 0 || dev >= 64) return (int)cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mapped_mu);
    if (!g_mapped[dev].host) {
        void* h = nullptr;
        if ((e = cudaHostAlloc(&h, 64, cudaHostAllocMapped | cudaHostAllocPortable)) != cudaSuccess) return (int)e;
        void* d = nullptr;
        if ((e = cudaHostGetDevicePointer(&d, h, 0)) != cudaSuccess) {
            cudaFreeHost(h);
            return (int)e;
        }
        memset(h, 0, 64);
        g_mapped[dev].host = static_cast<double*>(h);
        g_mapped[dev].dev = static_cast<double*>(d);
    }
    g_mapped[dev].seq += 1.0;
    *m = g_mapped[dev];
    return 0;
}

// Wait until the reduction's sequence number shows in slot ncomp: poll the mapped slot for up
// to 20 ms (results of small states arrive within microseconds), then synchronise the stream,
// which also reports any error of the launch.
int wait_mapped(const MappedOut& m, unsigned ncomp, cudaStream_t st) {
    volatile const double* flag = m.host + ncomp;
    const auto t0 = std::chrono::steady_clock::now();
    for (unsigned i = 0;; ++i) {
        if (*flag == m.seq) return 0;
        if ((i & 255u) == 255u && std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(20)) break;
    }
    const int rc = (int)cudaStreamSynchronize(st);
    if (rc) return rc;
    return *flag == m.seq ? 0 : (int)cudaErrorUnknown;
}

struct DevMemC2 {
    const double2* p;
    __device__ __forceinline__ double2 ld(idx_t i) const { return p[i]; }
};

__global__ void k_exp_table(const double* __restrict__ diag, idx_t dim, double t, double2* __restrict__ tab) {
    for (idx_t x = (idx_t)blockIdx.x * blockDim.x + threadIdx.x; x < dim; x += (idx_t)gridDim.x * blockDim.x) {
        double sn, cs;
        sincos(diag[x] * t, &sn, &cs);
        tab[x] = c2(cs, sn);
    }
}

}  // namespace

extern "C" {

int orkan_cu_fill(int layout, unsigned log_tile, void* data, unsigned n, double re, double im, void* stream) {
    if (!data || n > 62) return (int)cudaErrorInvalidValue;
    idx_t len;
    unsigned clt = 0;
    idx_t cdim = 0;
    const idx_t d = idx_t(1) << n;
    if (layout == 0) {
        len = d;
    } else if (layout == 1) {
        len = PackedMap{d}.len();
    } else if (layout == 2 && log_tile >= 1 && log_tile <= 8) {
        len = TiledMap{d, log_tile}.len();
        if (d < (idx_t(1) << log_tile)) { clt = log_tile; cdim = d; }
    } else {
        return (int)cudaErrorInvalidValue;
    }
    const unsigned grid = grid_for(kPureThreads * 4, len, kFullGrid);
    k_fill<<<grid, kPureThreads, 0, as_stream(stream)>>>(DevMem{static_cast<double2*>(data)}, len, c2(re, im), clt,
                                                         cdim);
    return finish_launch();
}

int orkan_cu_pure_gate1(void* psi, unsigned n, unsigned target, int op, double c, double s, void* stream) {
    if (!psi || n < 1 || n > 62 || target >= n || op < 0 || op >= kNumOp1) return (int)cudaErrorInvalidValue;
    const idx_t npairs = idx_t(1) << (n - 1);
    const unsigned grid = grid_for(kPureThreads * kVec, npairs, kFullGrid);
    DevMem mem{static_cast<double2*>(psi)};
    cudaStream_t st = as_stream(stream);
    switch (op) {
#define ORKAN_CASE1(OPC) \
    case OPC: k_pure1q<OPC><<<grid, kPureThreads, 0, st>>>(mem, npairs, target, c, s); break;
        ORKAN_CASE1(kOpX) ORKAN_CASE1(kOpY) ORKAN_CASE1(kOpZ) ORKAN_CASE1(kOpH) ORKAN_CASE1(kOpS)
        ORKAN_CASE1(kOpSdg) ORKAN_CASE1(kOpT) ORKAN_CASE1(kOpTdg) ORKAN_CASE1(kOpHy) ORKAN_CASE1(kOpRx)
        ORKAN_CASE1(kOpRy) ORKAN_CASE1(kOpRz) ORKAN_CASE1(kOpP)
#undef ORKAN_CASE1
        default: return (int)cudaErrorInvalidValue;
    }
    return finish_launch();
}

int orkan_cu_pure_gate2(void* psi, unsigned n, unsigned qa, unsigned qb, int op, void* stream) {
    if (!psi || n < 2 || n > 62 || qa >= n || qb >= n || qa == qb || op < 0 || op >= kNumOp2)
        return (int)cudaErrorInvalidValue;
    const idx_t nq = idx_t(1) << (n - 2);
    const unsigned grid = grid_for(kPureThreads * kVec, nq, kFullGrid);
    DevMem mem{static_cast<double2*>(psi)};
    cudaStream_t st = as_stream(stream);
    switch (op) {
        case kOpCX: k_pure2q<kOpCX><<<grid, kPureThreads, 0, st>>>(mem, nq, qa, qb); break;
        case kOpCY: k_pure2q<kOpCY><<<grid, kPureThreads, 0, st>>>(mem, nq, qa, qb); break;
        case kOpCZ: k_pure2q<kOpCZ><<<grid, kPureThreads, 0, st>>>(mem, nq, qa, qb); break;
        case kOpSwap: k_pure2q<kOpSwap><<<grid, kPureThreads, 0, st>>>(mem, nq, qa, qb); break;
        default: return (int)cudaErrorInvalidValue;
    }
    return finish_launch();
}

int orkan_cu_pure_ccx(void* psi, unsigned n, unsigned c1, unsigned c2q, unsigned t, void* stream) {
    if (!psi || n < 3 || n > 62 || c1 >= n || c2q >= n || t >= n || c1 == c2q || c1 == t || c2q == t)
        return (int)cudaErrorInvalidValue;
    const idx_t no = idx_t(1) << (n - 3);
    const unsigned grid = grid_for(kPureThreads * kVec, no, kFullGrid);
    k_pure_ccx<<<grid, kPureThreads, 0, as_stream(stream)>>>(DevMem{static_cast<double2*>(psi)}, no, c1, c2q, t);
    return finish_launch();
}

int orkan_cu_pure_fused(void* psi, unsigned n, unsigned log_chunk, unsigned ngates, const orkan_fgate_t* gates,
                        void* stream) {
    if (!psi || !gates) return (int)cudaErrorInvalidValue;
    FusedPlan plan;
    if (!fused_plan(n, log_chunk, ngates, gates, &plan)) return (int)cudaErrorInvalidValue;
    const size_t smem = fused_smem_bytes(plan);
    static std::atomic<bool> attr{false};
    if (!attr.load(std::memory_order_relaxed)) {
        cudaFuncSetAttribute(k_pure_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
        attr.store(true, std::memory_order_relaxed);
    }
    // threads per block: 128 (four blocks per SM at 124 registers; measured 15 % faster than
    // 256 on a 200-gate random circuit at 30 q), or 256 through the tuning knob
    // ORKAN_FUSE_THREADS, read once
    static const unsigned nt = [] {
        const char* e = getenv("ORKAN_FUSE_THREADS");
        return (e && atoi(e) == 256) ? kFuseThreads : 128u;
    }();
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pure_fused, (int)nt, smem) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const unsigned grid = grid_for(1, plan.nchunks(), (unsigned)(sm_count() * per_sm));
    k_pure_fused<<<grid, nt, smem, as_stream(stream)>>>(DevMem{static_cast<double2*>(psi)}, plan);
    return finish_launch();
}

unsigned long long orkan_cu_fused_need(const orkan_fgate_t* g) { return g ? fused_need(*g) : ~0ull; }

int orkan_cu_dm_unitary(int layout, unsigned log_tile, void* rho, unsigned n, unsigned k, const unsigned* qubits,
                        const double* u, void* stream) {
    if (!rho || !qubits || !u || !layout_ok(layout, log_tile) || (k != 1 && k != 2) || n > 40)
        return (int)cudaErrorInvalidValue;
    DmGeom g;
    if (!dm_geometry(n, k, qubits, ls_max_for(layout, log_tile), &g, dm_max_v_low())) return (int)cudaErrorInvalidValue;
    if (k == 1) {
        OpMix1 op;
        for (unsigned i = 0; i < 4; ++i) op.u[i] = ld_c(u, i);
        return launch_engine_map(layout, log_tile, rho, n, g, op, as_stream(stream));
    }
    OpMix2 op;
    for (unsigned i = 0; i < 16; ++i) op.u[i] = ld_c(u, i);
    return launch_engine_map(layout, log_tile, rho, n, g, op, as_stream(stream));
}

int orkan_cu_dm_monomial(int layout, unsigned log_tile, void* rho, unsigned n, unsigned k, const unsigned* qubits,
                         const unsigned* src, const double* phase, void* stream) {
    if (!rho || !qubits || !src || !phase || !layout_ok(layout, log_tile) || k < 1 || k > 3 || n > 40)
        return (int)cudaErrorInvalidValue;
    OpMonomial op;
    const unsigned m = 1u << k;
    for (unsigned y = 0; y < 8; ++y) { op.src[y] = y; op.phase[y] = c2(1.0, 0.0); }
    for (unsigned y = 0; y < m; ++y) {
        if (src[y] >= m || src[src[y]] != y) return (int)cudaErrorInvalidValue;   // must be an involution
        op.src[y] = src[y];
        op.phase[y] = ld_c(phase, y);
    }
    DmGeom g;
    if (!dm_monomial_setup(n, k, qubits, op, ls_max_for(layout, log_tile), dm_max_v_low(), &g))
        return (int)cudaErrorInvalidValue;
    return launch_engine_map(layout, log_tile, rho, n, g, op, as_stream(stream));
}

int orkan_cu_dm_phase(int layout, unsigned log_tile, void* rho, unsigned n, unsigned k, const unsigned* qubits,
                      const double* phase, void* stream) {
    if (!rho || !qubits || !phase || !layout_ok(layout, log_tile) || k < 1 || k > 3 || n > 40)
        return (int)cudaErrorInvalidValue;
    for (unsigned j = 0; j < k; ++j)
        if (qubits[j] >= n) return (int)cudaErrorInvalidValue;
    if (k == 1 && phase[0] == 1.0 && phase[1] == 0.0) {
        GateFactor1 f1;
        f1.q = qubits[0];
        f1.ph1 = ld_c(phase, 1);
        return launch_phase(layout, log_tile, rho, n, f1, as_stream(stream));
    }
    {                                                   // controlled phase (CZ): a mask test per element
        bool ctrl = true;
        for (unsigned y = 0; y + 1 < (1u << k); ++y) ctrl = ctrl && phase[2 * y] == 1.0 && phase[2 * y + 1] == 0.0;
        if (ctrl) {
            GateFactorCtrl fc;
            fc.mask = 0;
            for (unsigned j = 0; j < k; ++j) fc.mask |= 1ull << qubits[j];
            fc.ph = ld_c(phase, (1u << k) - 1);
            return launch_phase(layout, log_tile, rho, n, fc, as_stream(stream));
        }
    }
    GateFactor fac;
    fac.k = k;
    for (unsigned j = 0; j < 3; ++j) fac.q[j] = j < k ? qubits[j] : 0;
    for (unsigned y = 0; y < 8; ++y) fac.phase[y] = y < (1u << k) ? ld_c(phase, y) : c2(1.0, 0.0);
    return launch_phase(layout, log_tile, rho, n, fac, as_stream(stream));
}

int orkan_cu_dm_superop1(int layout, unsigned log_tile, void* rho, unsigned n, unsigned target, const double* sop,
                         void* stream) {
    if (!rho || !sop || !layout_ok(layout, log_tile) || target >= n || n > 40) return (int)cudaErrorInvalidValue;
    OpSuper1 op;
    for (unsigned i = 0; i < 16; ++i) op.s[i] = ld_c(sop, i);
    DmGeom g;
    const unsigned q[1] = {target};
    if (!dm_geometry(n, 1, q, ls_max_for(layout, log_tile), &g, dm_max_v_low())) return (int)cudaErrorInvalidValue;
    return launch_engine_map(layout, log_tile, rho, n, g, op, as_stream(stream));
}

int orkan_cu_dm_superop2(int layout, unsigned log_tile, void* rho, unsigned n, unsigned q0, unsigned q1,
                         const double* sop, void* stream) {
    if (!rho || !sop || !layout_ok(layout, log_tile) || q0 >= n || q1 >= n || q0 == q1 || n > 40)
        return (int)cudaErrorInvalidValue;
    OpSuper2 op;
    for (unsigned i = 0; i < 256; ++i) op.s[i] = ld_c(sop, i);
    DmGeom g;
    const unsigned q[2] = {q0, q1};
    if (!dm_geometry(n, 2, q, ls_max_for(layout, log_tile), &g, dm_max_v_low())) return (int)cudaErrorInvalidValue;
    return launch_engine_map(layout, log_tile, rho, n, g, op, as_stream(stream));
}

int orkan_cu_exp_diag(int layout, unsigned log_tile, void* data, unsigned n, const double* diag, double t,
                      void* stream) {
    if (!data || !diag || n > 62) return (int)cudaErrorInvalidValue;
    if (t == 0.0) return 0;
    cudaStream_t st = as_stream(stream);
    const idx_t d = idx_t(1) << n;
    if (layout == 0) {
        const unsigned grid = grid_for(kPureThreads * kVec, d, kFullGrid);
        k_pure_exp_diag<<<grid, kPureThreads, 0, st>>>(DevMem{static_cast<double2*>(data)}, DevMemR{diag}, d, t);
        return finish_launch();
    }
    if (!layout_ok(layout, log_tile) || n > 40) return (int)cudaErrorInvalidValue;
    double2* tab = static_cast<double2*>(scratch_get(d * sizeof(double2)));
    if (!tab) return (int)cudaErrorMemoryAllocation;
    const unsigned grid = grid_for(256, d, kFullGrid);
    k_exp_table<<<grid, 256, 0, st>>>(diag, d, t, tab);
    const int rc = finish_launch();
    if (rc) return rc;
    TableFactor<DevMemC2> fac{DevMemC2{tab}};
    return launch_phase(layout, log_tile, data, n, fac, st);
}

int orkan_cu_mean(int layout, unsigned log_tile, const void* data, unsigned n, const double* obs, double* result,
                  void* stream) {
    if (!data || !obs || !result || n > 62) return (int)cudaErrorInvalidValue;
    if (layout != 0 && !layout_ok(layout, log_tile)) return (int)cudaErrorInvalidValue;
    cudaStream_t st = as_stream(stream);
    const idx_t d = idx_t(1) << n;
    // PURE: 4 amplitudes per thread per block at least; DM: one diagonal element per thread
    const unsigned np = grid_for(layout == 0 ? kRedThreads * 4 : kRedThreads, d, kRedBlocks);
    double* part = static_cast<double*>(scratch_get(np * sizeof(double)));
    if (!part) return (int)cudaErrorMemoryAllocation;
    MappedOut out;
    int rc = mapped_out(&out);
    if (rc) return rc;
    const double2* rho = static_cast<const double2*>(data);
    if (layout == 0)
        k_mean_pure<<<np, kRedThreads, 0, st>>>(rho, obs, d, part, out.dev, out.seq);
    else if (layout == 1)
        k_mean_dm<PackedMap><<<np, kRedThreads, 0, st>>>(rho, PackedMap{d}, obs, part, out.dev, out.seq);
    else
        k_mean_dm<TiledMap><<<np, kRedThreads, 0, st>>>(rho, TiledMap{d, log_tile}, obs, part, out.dev, out.seq);
    if ((rc = finish_launch())) return rc;
    if ((rc = wait_mapped(out, 1, st))) return rc;
    *result = static_cast<volatile const double*>(out.host)[0];
    return 0;
}

int orkan_cu_matel_diag(const void* bra, const void* ket, unsigned n, const double* obs, double* result,
                        void* stream) {
    if (!bra || !ket || !obs || !result || n > 62) return (int)cudaErrorInvalidValue;
    cudaStream_t st = as_stream(stream);
    const idx_t d = idx_t(1) << n;
    const unsigned np = grid_for(kRedThreads * 4, d, kRedBlocks);
    double* part = static_cast<double*>(scratch_get(2 * np * sizeof(double)));
    if (!part) return (int)cudaErrorMemoryAllocation;
    MappedOut out;
    int rc = mapped_out(&out);
    if (rc) return rc;
    k_matel_pure<<<np, kRedThreads, 0, st>>>(static_cast<const double2*>(bra), static_cast<const double2*>(ket), obs,
                                             d, part, out.dev, out.seq);
    if ((rc = finish_launch())) return rc;
    if ((rc = wait_mapped(out, 2, st))) return rc;
    result[0] = static_cast<volatile const double*>(out.host)[0];
    result[1] = static_cast<volatile const double*>(out.host)[1];
    return 0;
}

unsigned long long orkan_cu_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

// Error word of the density-matrix engine (non-zero: a wait for staged data ran out).
unsigned orkan_cu_engine_status(void) {
    unsigned v = 0;
    if (cudaMemcpyFromSymbol(&v, g_dm_engine_error, sizeof(v)) != cudaSuccess) return 0xffffffffu;
    return v;
}

int orkan_cu_engine_status_clear(void) {
    const unsigned zero = 0;
    return (int)cudaMemcpyToSymbol(g_dm_engine_error, &zero, sizeof(zero));
}

void orkan_cu_engine_test_wait(unsigned long long polls, int drop_loads) {
    g_engine_test_drop.store(polls && drop_loads ? 1u : 0u, std::memory_order_relaxed);
    g_engine_test_polls.store(polls, std::memory_order_relaxed);
}

}  // extern "C"
