// scratch.cu - see scratch.cuh.
#include "scratch.cuh"

#include <mutex>

namespace orkan {

namespace {
constexpr int kMaxDev = 64;
constexpr int kSlots = 2;
std::mutex g_mu;
void* g_ptr[kMaxDev][kSlots] = {};
size_t g_size[kMaxDev][kSlots] = {};
}  // namespace

void* scratch_get_slot(int slot, size_t bytes) {
    int dev = 0;
    if (slot < 0 || slot >= kSlots || cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return nullptr;
    if (bytes == 0) bytes = 256;
    std::lock_guard<std::mutex> lock(g_mu);
    if (g_size[dev][slot] >= bytes) return g_ptr[dev][slot];
    if (g_ptr[dev][slot]) {
        cudaFree(g_ptr[dev][slot]);
        g_ptr[dev][slot] = nullptr;
        g_size[dev][slot] = 0;
    }
    size_t want = bytes + bytes / 4;   // headroom so slowly growing requests reallocate rarely
    want = (want + 4095) & ~size_t(4095);
    void* p = nullptr;
    if (cudaMalloc(&p, want) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    g_ptr[dev][slot] = p;
    g_size[dev][slot] = want;
    return p;
}

}  // namespace orkan

extern "C" void* orkan_internal_staging(size_t bytes) { return orkan::scratch_get_slot(1, bytes); }
