// noalloc.cu - exp_diag without any device allocation by the library.
//
// orkan_cu_exp_diag stages the per-index phase table of a density matrix in a scratch
// buffer that the library allocates (and, when a larger state arrives, frees and
// allocates again).  Some callers cannot allow that: a host program that hands nearly all
// device memory to its own pool allocator up front (as machine-learning frameworks do) has
// no room left for a stray cudaMalloc, and a latency-sensitive caller cannot absorb the
// device-wide wait that cudaFree performs when the buffer grows.  This entry point keeps
// the table in a fixed, file-scope device array instead, so it never allocates or frees.
//
// Limits and sharing: the table holds kNoAllocMaxDim = 65536 entries (1 MiB), enough for
// density matrices of up to 16 qubits; larger ones are rejected.  The array exists once per
// device for as long as the library stays loaded, every call on that device uses it, and
// it keeps the contents of the last call (each call overwrites the 2^n entries it uses, so
// nothing has to start at zero).  Two calls whose kernels overlap on the GPU (for example
// on different streams) race on the table.
#include "common.cuh"
#include "dm_phase.cuh"
#include "launch.cuh"

#include "../../../include/orkan_cu.h"

#include <mutex>
#include <stdio.h>

using namespace orkan;

namespace {

constexpr idx_t kNoAllocMaxDim = idx_t(1) << 16;
constexpr int kMaxDevices = 64;

// The table: one per device, alive until the library is unloaded.
static __device__ __align__(256) double2 g_noalloc_table[kNoAllocMaxDim];

// Device address of g_noalloc_table, resolved once per device by the first call made on
// that device (host code cannot use the symbol itself as a device pointer).  The mutex
// serialises first calls made from several host threads at once.
std::mutex g_table_mu;
double2* g_table_addr[kMaxDevices] = {};

struct TabMem {
    const double2* p;
    __device__ __forceinline__ double2 ld(idx_t i) const { return p[i]; }
};

__global__ void k_noalloc_table(const double* __restrict__ diag, idx_t dim, double t, double2* __restrict__ tab) {
    for (idx_t x = (idx_t)blockIdx.x * blockDim.x + threadIdx.x; x < dim; x += (idx_t)gridDim.x * blockDim.x) {
        double sn, cs;
        sincos(diag[x] * t, &sn, &cs);
        tab[x] = c2(cs, sn);
    }
}

int table_address(double2** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return (int)e;
    if (dev < 0 || dev >= kMaxDevices) return (int)cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_table_mu);
    if (!g_table_addr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_table);
        if (e != cudaSuccess) return (int)e;
        g_table_addr[dev] = static_cast<double2*>(ptr);
    }
    *out = g_table_addr[dev];
    return 0;
}

}  // namespace

extern "C" int orkan_cu_exp_diag_noalloc(int layout, unsigned log_tile, void* data, unsigned n, const double* diag,
                                         double t, void* stream) {
    if (!data || !diag || (layout != 1 && layout != 2) || (layout == 2 && (log_tile < 1 || log_tile > 8)))
        return (int)cudaErrorInvalidValue;
    const idx_t d = n < 63 ? idx_t(1) << n : 0;
    if (d == 0 || d > kNoAllocMaxDim) {
        fprintf(stderr, "orkan: orkan_cu_exp_diag_noalloc: %u qubits need a %llu-entry phase table; "
                        "the fixed device table holds %llu (at most 16 qubits)\n",
                n, (unsigned long long)(n < 63 ? d : 0), (unsigned long long)kNoAllocMaxDim);
        return (int)cudaErrorInvalidValue;
    }
    if (t == 0.0) return 0;
    double2* tab = nullptr;
    int rc = table_address(&tab);
    if (rc) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    k_noalloc_table<<<grid_for(256, d, (unsigned)sm_count() * 8u), 256, 0, st>>>(diag, d, t, tab);
    rc = finish_launch();
    if (rc) return rc;
    return launch_phase(layout, log_tile, data, n, TableFactor<TabMem>{TabMem{tab}}, st);
}
