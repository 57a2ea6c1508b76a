// reduce.cuh - deterministic reductions for mean and matel_diag.
//
// Reference: mean_pure / matel_diag_pure (src/meas/meas_pure.c:20-46), mean_packed
// (meas_packed.c:23-51, diagonal at stride d, d-1, ...), mean_tiled (meas_tiled.c:29-69,
// diagonal tiles at stride TILE_DIM+1).
//
// Every reduction uses a fixed partition (up to kRedBlocks contiguous chunks, a fixed
// per-thread order, a fixed shuffle tree) and writes one partial per block to a scratch
// array; the block that finishes last (a ticket counter taken after a memory fence) folds
// the partials in index order and resets the counter, all in one launch.  Which block
// folds does not change the order of the fold, so results are bit-identical from run to
// run.  The density-matrix mean reads only the d diagonal elements, spread over blocks
// of kRedThreads elements each.
#pragma once

#include "common.cuh"

namespace orkan {

constexpr unsigned kRedThreads = 256;
constexpr unsigned kRedBlocks = 4736;      // fixed number of partial sums (32 per SM of B200)

#ifdef __CUDACC__
template <unsigned NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    v = 0.0;
    if (warp == 0) {
        v = lane < NT / 32 ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;
}

// Ticket counters of the one-launch reductions (zero at load; the folding block resets its
// counter, so every launch starts from zero).  Calls are stream-ordered on one device.
static __device__ unsigned g_red_ticket[3];

// Is this block the last of the grid to finish its partial?  Thread 0 wrote the block's
// partial before the call.
__device__ __forceinline__ bool last_block_done(unsigned* ticket) {
    __shared__ bool last;
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    return last;
}

// out[c] = sum_b partial[b * ncomp + c] in fixed order, by the whole block; then out[ncomp] =
// seq, written after the results are visible system-wide (out may be mapped host memory the
// host polls); resets the ticket.
__device__ __forceinline__ void fold_partials(const double* partial, unsigned np, unsigned ncomp, double* out,
                                              unsigned* ticket, double seq) {
    __shared__ double sh[32];
    __threadfence();
    for (unsigned c = 0; c < ncomp; ++c) {
        double acc = 0.0;
        for (unsigned b = threadIdx.x; b < np; b += kRedThreads) acc += __ldcg(partial + b * ncomp + c);
        acc = block_sum<kRedThreads>(acc, sh);
        if (threadIdx.x == 0) out[c] = acc;
    }
    if (threadIdx.x == 0) {
        __threadfence_system();          // the results land before the sequence number
        volatile double* vs = out + ncomp;
        *vs = seq;
        *ticket = 0u;
    }
}

// partial[b] = sum over chunk b of obs[x] * |psi_x|^2; the last block folds them into out[0]
__global__ void __launch_bounds__(kRedThreads) k_mean_pure(const double2* __restrict__ psi,
                                                           const double* __restrict__ obs, idx_t dim,
                                                           double* __restrict__ partial, double* __restrict__ out, double seq) {
    __shared__ double sh[32];
    const idx_t chunk = (dim + gridDim.x - 1) / gridDim.x;
    const idx_t begin = (idx_t)blockIdx.x * chunk;
    const idx_t end = begin + chunk < dim ? begin + chunk : dim;
    double acc = 0.0;
    idx_t x = begin + threadIdx.x;
    for (; x + 3 * kRedThreads < end; x += 4 * kRedThreads) {
        double2 a[4];
        double o[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) { a[u] = psi[x + u * kRedThreads]; o[u] = __ldg(obs + x + u * kRedThreads); }
#pragma unroll
        for (int u = 0; u < 4; ++u) acc += o[u] * (a[u].x * a[u].x + a[u].y * a[u].y);
    }
    for (; x < end; x += kRedThreads) {
        const double2 a = psi[x];
        acc += __ldg(obs + x) * (a.x * a.x + a.y * a.y);
    }
    acc = block_sum<kRedThreads>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
    if (last_block_done(&g_red_ticket[0])) fold_partials(partial, gridDim.x, 1, out, &g_red_ticket[0], seq);
}

// re/im partials of sum_x obs[x] conj(bra_x) ket_x
__global__ void __launch_bounds__(kRedThreads) k_matel_pure(const double2* __restrict__ bra,
                                                            const double2* __restrict__ ket,
                                                            const double* __restrict__ obs, idx_t dim,
                                                            double* __restrict__ partial, double* __restrict__ out, double seq) {
    __shared__ double sh[32];
    const idx_t chunk = (dim + gridDim.x - 1) / gridDim.x;
    const idx_t begin = (idx_t)blockIdx.x * chunk;
    const idx_t end = begin + chunk < dim ? begin + chunk : dim;
    double sre = 0.0, sim = 0.0;
    idx_t x = begin + threadIdx.x;
    for (; x + 3 * kRedThreads < end; x += 4 * kRedThreads) {
        double2 a[4], b[4];
        double o[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a[u] = bra[x + u * kRedThreads];
            b[u] = ket[x + u * kRedThreads];
            o[u] = __ldg(obs + x + u * kRedThreads);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            sre += o[u] * (a[u].x * b[u].x + a[u].y * b[u].y);
            sim += o[u] * (a[u].x * b[u].y - a[u].y * b[u].x);
        }
    }
    for (; x < end; x += kRedThreads) {
        const double2 a = bra[x], b = ket[x];
        const double o = __ldg(obs + x);
        sre += o * (a.x * b.x + a.y * b.y);
        sim += o * (a.x * b.y - a.y * b.x);
    }
    sre = block_sum<kRedThreads>(sre, sh);
    sim = block_sum<kRedThreads>(sim, sh);
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = sre; partial[2 * blockIdx.x + 1] = sim; }
    if (last_block_done(&g_red_ticket[1])) fold_partials(partial, gridDim.x, 2, out, &g_red_ticket[1], seq);
}

// sum_x obs[x] * Re rho_xx over the diagonal of a packed or tiled density matrix:
// block b sums a contiguous run of diagonal indices, the last block folds.
template <class Map>
__global__ void __launch_bounds__(kRedThreads) k_mean_dm(const double2* __restrict__ rho, Map map,
                                                         const double* __restrict__ obs, double* __restrict__ partial,
                                                         double* __restrict__ out, double seq) {
    __shared__ double sh[32];
    const idx_t chunk = (map.d + gridDim.x - 1) / gridDim.x;
    const idx_t begin = (idx_t)blockIdx.x * chunk;
    const idx_t end = begin + chunk < map.d ? begin + chunk : map.d;
    double acc = 0.0;
    idx_t x = begin + threadIdx.x;
    for (; x + 3 * kRedThreads < end; x += 4 * kRedThreads) {
        double v[4], o[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            v[u] = rho[map.at(x + u * kRedThreads, x + u * kRedThreads)].x;
            o[u] = __ldg(obs + x + u * kRedThreads);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) acc += o[u] * v[u];
    }
    for (; x < end; x += kRedThreads) acc += __ldg(obs + x) * rho[map.at(x, x)].x;
    acc = block_sum<kRedThreads>(acc, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
    if (last_block_done(&g_red_ticket[2])) fold_partials(partial, gridDim.x, 1, out, &g_red_ticket[2], seq);
}
#endif

}  // namespace orkan
