// sample.cu - device building blocks of sample_matrix (include/orkan_sample.h): the
// weighted accumulation of a channel sum, and blocks of S = Phi_i^H diag(obs) Phi_j.
//
// The operation is specified by the reference (docs/SAMPLE_MATRIX.md sections 1-6) and not
// implemented there.  Its recommended algorithm forms each block with a BLAS zgemm on
// Y = obs * Phi_j; here a block of at most 16 x 16 columns is one kernel that stages 64
// amplitudes of every column (and of obs) in shared memory and lets each thread own one
// (i, j) pair, so obs * Phi_j is never written out.  The amplitude range is cut into a
// fixed number of slices whose partial sums are added in slice order by a second kernel:
// an entry does not depend on the block shape it is computed in.
#include "common.cuh"

#include "../../../include/orkan_cu.h"

#include <cuda_runtime.h>

namespace orkan {
namespace {

constexpr unsigned kSmTile = 16;        // columns per side of one block
constexpr unsigned kSmSlices = 512;     // fixed partition of the amplitude range
constexpr unsigned kSmChunk = 64;       // amplitudes staged per step
constexpr unsigned kSmThreads = kSmTile * kSmTile;

__global__ void __launch_bounds__(256) k_lincomb(double2* acc, const double2* x, double2 w, idx_t len, int first) {
    const idx_t stride = (idx_t)gridDim.x * blockDim.x;
    for (idx_t i = (idx_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride) {
        const double2 t = cmul(w, x[i]);
        acc[i] = first ? t : cadd(acc[i], t);
    }
}

// Slice s of the amplitudes: partial[s][i * 16 + j] = sum over the slice, in order, of
// conj(phi_i[x]) obs[x] phi_j[x].
__global__ void __launch_bounds__(kSmThreads) k_sm_partial(const double2* pi, unsigned bi, const double2* pj,
                                                           unsigned bj, idx_t len, const double* obs,
                                                           double2* partial) {
    __shared__ double2 si[kSmChunk][kSmTile + 1], sj[kSmChunk][kSmTile + 1];
    __shared__ double sh[kSmChunk];
    const unsigned t = threadIdx.x, i = t / kSmTile, j = t % kSmTile;
    const idx_t per = ((len + kSmSlices - 1) / kSmSlices + kSmChunk - 1) / kSmChunk * kSmChunk;
    const idx_t x0 = (idx_t)blockIdx.x * per;
    const idx_t x1 = x0 + per < len ? x0 + per : len;
    const bool active = i < bi && j < bj;
    double re = 0.0, im = 0.0;
    for (idx_t xb = x0; xb < x1; xb += kSmChunk) {
        const unsigned m = (unsigned)(x1 - xb < kSmChunk ? x1 - xb : kSmChunk);
        for (unsigned e = t; e < bi * kSmChunk; e += kSmThreads) {
            const unsigned c = e / kSmChunk, x = e % kSmChunk;
            si[x][c] = x < m ? pi[(idx_t)c * len + xb + x] : c2(0.0, 0.0);
        }
        for (unsigned e = t; e < bj * kSmChunk; e += kSmThreads) {
            const unsigned c = e / kSmChunk, x = e % kSmChunk;
            sj[x][c] = x < m ? pj[(idx_t)c * len + xb + x] : c2(0.0, 0.0);
        }
        if (t < kSmChunk) sh[t] = t < m ? obs[xb + t] : 0.0;
        __syncthreads();
        if (active) {
            for (unsigned x = 0; x < m; ++x) {
                const double2 a = si[x][i], b = sj[x][j];
                const double h = sh[x];
                re += h * (a.x * b.x + a.y * b.y);
                im += h * (a.x * b.y - a.y * b.x);
            }
        }
        __syncthreads();
    }
    partial[(idx_t)blockIdx.x * kSmThreads + t] = c2(re, im);
}

__global__ void __launch_bounds__(kSmThreads) k_sm_fold(const double2* partial, unsigned bi, unsigned bj,
                                                        double2* out) {
    const unsigned t = threadIdx.x, i = t / kSmTile, j = t % kSmTile;
    if (i >= bi || j >= bj) return;
    double re = 0.0, im = 0.0;
    for (unsigned s = 0; s < kSmSlices; ++s) {
        const double2 v = partial[(idx_t)s * kSmThreads + t];
        re += v.x;
        im += v.y;
    }
    out[i + (idx_t)j * bi] = c2(re, im);
}

}  // namespace
}  // namespace orkan

using namespace orkan;

extern "C" {

int orkan_cu_lincomb(void* acc, const void* x, double w_re, double w_im, unsigned long long len, int first,
                     void* stream) {
    if (!acc || !x || len == 0) return (int)cudaErrorInvalidValue;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const idx_t want = (len + 255) / 256, cap = (idx_t)sms * 8;
    const unsigned grid = (unsigned)(want < cap ? want : cap);
    k_lincomb<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<double2*>(acc), static_cast<const double2*>(x), c2(w_re, w_im), (idx_t)len, first);
    return (int)cudaGetLastError();
}

size_t orkan_cu_sm_scratch_bytes(void) { return (size_t)kSmSlices * kSmThreads * sizeof(double2); }

int orkan_cu_sm_block(const void* phi_i, unsigned bi, const void* phi_j, unsigned bj, unsigned long long len,
                      const double* obs, void* out, void* scratch, void* stream) {
    if (!phi_i || !phi_j || !obs || !out || !scratch || len == 0 || bi < 1 || bj < 1 || bi > kSmTile ||
        bj > kSmTile)
        return (int)cudaErrorInvalidValue;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double2* partial = static_cast<double2*>(scratch);
    k_sm_partial<<<kSmSlices, kSmThreads, 0, st>>>(static_cast<const double2*>(phi_i), bi,
                                                   static_cast<const double2*>(phi_j), bj, (idx_t)len, obs, partial);
    k_sm_fold<<<1, kSmThreads, 0, st>>>(partial, bi, bj, static_cast<double2*>(out));
    return (int)cudaGetLastError();
}

}  // extern "C"
