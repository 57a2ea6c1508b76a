// mlp.cu - FP32 surrogate network of include/orkan_mlp.h: tiled GEMMs with fused bias/GELU
// epilogues, deterministic reductions, Adam, minibatch gather, a captured training step and
// input-space ascent for proposals.  Everything runs in the caller's stream.
#include "../../../include/orkan_mlp.h"

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <vector>

namespace {

std::atomic<unsigned long long> g_launches{0};

constexpr int kBM = 64, kBN = 64, kBK = 16, kGemmThreads = 256;   // default tile; 32 x 32 for small grids
constexpr float kInvSqrt2 = 0.70710678118654752440f;
constexpr float kInvSqrt2Pi = 0.39894228040143267794f;

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * kInvSqrt2)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * kInvSqrt2)) + z * kInvSqrt2Pi * expf(-0.5f * z * z);
}

enum Epi : int { kEpiStore = 0, kEpiBiasGelu = 1, kEpiGeluBack = 2 };

// C[m][n] = sum_k opA[m][k] opB[k][n];  opA[m][k] = TA ? A[k][m] : A[m][k],
// opB[k][n] = TB ? B[n][k] : B[k][n] (row-major with leading dimensions lda, ldb).
// Epilogues: store; z = acc + bias[n] into C and gelu(z) into out2; acc * gelu'(aux[m][n]).
// Each output is one thread's fixed-order sum over k, so results are deterministic.
template <bool TA, bool TB, int EPI, int kBM = 64, int kBN = 64>
__global__ void __launch_bounds__(kGemmThreads) k_gemm(int M, int N, int K, const float* __restrict__ A, int lda,
                                                       const float* __restrict__ B, int ldb, float* __restrict__ C,
                                                       int ldc, const float* __restrict__ bias,
                                                       const float* __restrict__ aux, float* __restrict__ out2) {
    constexpr int TM = kBM / 16, TN = kBN / 16;          // outputs per thread: TM x TN
    __shared__ float As[kBK][kBM + 4];
    __shared__ float Bs[kBK][kBN + 4];
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
    // split over k (gridDim.z slices of whole kBK tiles): slice z sums its own k range and
    // stores to its own M x ldc plane of C
    const int ktiles = (K + kBK - 1) / kBK, per = (ktiles + gridDim.z - 1) / gridDim.z;
    const int kbeg = blockIdx.z * per * kBK, kend = min(K, (int)(blockIdx.z + 1) * per * kBK);
    C += (size_t)blockIdx.z * M * ldc;
    float acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = 0.f;
    for (int k0 = kbeg; k0 < kend; k0 += kBK) {
        for (int e = threadIdx.x; e < kBM * kBK; e += kGemmThreads) {
            const int mm = TA ? e % kBM : e / kBK, kk = TA ? e / kBM : e % kBK;
            const int gm = m0 + mm, gk = k0 + kk;
            float v = 0.f;
            if (gm < M && gk < kend) v = TA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk];
            As[kk][mm] = v;
        }
        for (int e = threadIdx.x; e < kBN * kBK; e += kGemmThreads) {
            const int nn = TB ? e / kBK : e % kBN, kk = TB ? e % kBK : e / kBN;
            const int gn = n0 + nn, gk = k0 + kk;
            float v = 0.f;
            if (gn < N && gk < kend) v = TB ? B[(size_t)gn * ldb + gk] : B[(size_t)gk * ldb + gn];
            Bs[kk][nn] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kBK; ++kk) {
            float a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int m = m0 + ty + 16 * i, n = n0 + tx + 16 * j;
            if (m >= M || n >= N) continue;
            const size_t o = (size_t)m * ldc + n;
            if (EPI == kEpiStore) {
                C[o] = acc[i][j];
            } else if (EPI == kEpiBiasGelu) {
                const float z = acc[i][j] + bias[n];
                C[o] = z;
                out2[o] = gelu(z);
            } else {
                C[o] = acc[i][j] * gelu_grad(aux[o]);
            }
        }
}

// out[i] = sum over the slices z < nz of part[z * count + i], in slice order.
__global__ void k_sum_slices(const float* __restrict__ part, int nz, size_t count, float* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float s = 0.f;
    for (int z = 0; z < nz; ++z) s += part[(size_t)z * count + i];
    out[i] = s;
}

// y[b] = sum_h A[b][h] w[h] + w0, one warp per row, fixed shuffle tree.
__global__ void k_rowdot(const float* __restrict__ A, int rows, int h, const float* __restrict__ w,
                         const float* __restrict__ w0, float* __restrict__ y) {
    const int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x % 32;
    if (row >= rows) return;
    float s = 0.f;
    for (int k = lane; k < h; k += 32) s = fmaf(A[(size_t)row * h + k], w[k], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) y[row] = s + w0[0];
}

// dy[b] = 2 (y[b] - t[b]) / batch (or 1 when t is NULL: the gradient of f itself);
// loss_slot[0] = mean squared error (one block, fixed order).
__global__ void k_loss(const float* __restrict__ y, const float* __restrict__ t, int batch, float* __restrict__ dy,
                       float* __restrict__ loss_slot) {
    __shared__ float red[1024];
    float s = 0.f;
    for (int b = threadIdx.x; b < batch; b += blockDim.x) {
        if (t) {
            const float d = y[b] - t[b];
            dy[b] = 2.0f * d / (float)batch;
            s = fmaf(d, d, s);
        } else {
            dy[b] = 1.0f;
        }
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss_slot) loss_slot[0] = red[0] / (float)batch;
}

// out[n] = sum_m X[m][n] (fixed order over m), and optionally out[n] for a column vector.
__global__ void k_colsum(const float* __restrict__ X, int rows, int cols, float* __restrict__ out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= cols) return;
    float s = 0.f;
    for (int m = 0; m < rows; ++m) s += X[(size_t)m * cols + n];
    out[n] = s;
}

// dW3[h] = sum_b A2[b][h] dy[b]
__global__ void k_coldot(const float* __restrict__ X, int rows, int cols, const float* __restrict__ v,
                         float* __restrict__ out) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= cols) return;
    float s = 0.f;
    for (int m = 0; m < rows; ++m) s = fmaf(X[(size_t)m * cols + n], v[m], s);
    out[n] = s;
}

// dZ2[b][h] = dy[b] w3[h] gelu'(Z2[b][h])
__global__ void k_outer_gelu(const float* __restrict__ dy, const float* __restrict__ w, const float* __restrict__ Z,
                             int rows, int cols, float* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)rows * cols) return;
    const int b = (int)(i / cols), h = (int)(i % cols);
    out[i] = dy[b] * w[h] * gelu_grad(Z[i]);
}

__global__ void k_step_begin(unsigned* step) {
    ++step[0];
    ++step[1];
}

// Adam with bias correction at step t = step[0] (1-based, all steps of the network).
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, size_t count, float lr, const unsigned* __restrict__ step) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float t = (float)step[0];
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float mi = b1 * m1[i] + (1.0f - b1) * g[i];
    const float vi = b2 * m2[i] + (1.0f - b2) * g[i] * g[i];
    m1[i] = mi;
    m2[i] = vi;
    const float mh = mi / (1.0f - powf(b1, t)), vh = vi / (1.0f - powf(b2, t));
    p[i] -= lr * mh / (sqrtf(vh) + eps);
}

// Adam ascent on inputs, clamped to [lo, hi].
__global__ void k_adam_inputs(float* __restrict__ x, const float* __restrict__ g, float* __restrict__ m1,
                              float* __restrict__ m2, size_t count, float lr, int t, float lo, float hi) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float mi = b1 * m1[i] + (1.0f - b1) * g[i];
    const float vi = b2 * m2[i] + (1.0f - b2) * g[i] * g[i];
    m1[i] = mi;
    m2[i] = vi;
    const float mh = mi / (1.0f - powf(b1, (float)t)), vh = vi / (1.0f - powf(b2, (float)t));
    x[i] = fminf(hi, fmaxf(lo, x[i] + lr * mh / (sqrtf(vh) + eps)));
}

__host__ __device__ inline uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__host__ __device__ inline uint64_t gcd64(uint64_t a, uint64_t b) {
    while (b) { const uint64_t t = a % b; a = b; b = t; }
    return a;
}

// Minibatch of the current step (schedule counter step[1], 1-based): epoch e = (s - 1) / spe,
// position j = (s - 1) % spe; sample i of the epoch is (a_e i + c_e) mod count.
__global__ void k_gather(const float* __restrict__ X, const float* __restrict__ T, unsigned count, int n_in, int batch,
                         unsigned spe, uint64_t seed, const unsigned* __restrict__ step, float* __restrict__ xb,
                         float* __restrict__ tb) {
    const unsigned s = step[1] - 1, e = s / spe, j = s % spe;
    uint64_t a = mix64(seed ^ (0x5851f42d4c957f2dull * (e + 1))) % count;
    if (a == 0) a = 1;
    while (gcd64(a, count) != 1) a = (a + 1) % count == 0 ? 1 : a + 1;
    const uint64_t c = mix64(seed + 0x632be59bd9b4e019ull * (e + 1)) % count;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < batch; r += gridDim.x * blockDim.x) {
        const uint64_t i = (uint64_t)j * batch + r;
        const uint64_t src = (a * i + c) % count;
        for (int k = 0; k < n_in; ++k) xb[(size_t)r * n_in + k] = X[src * n_in + k];
        tb[r] = T[src];
    }
}

// Mean of the per-step losses of the last epoch.
__global__ void k_epoch_loss(const float* __restrict__ losses, unsigned spe, float* __restrict__ out) {
    float s = 0.f;
    for (unsigned k = 0; k < spe; ++k) s += losses[k];
    out[0] = s / (float)spe;
}

__global__ void k_copy_loss(const float* __restrict__ src, const unsigned* __restrict__ step, unsigned spe,
                            float* __restrict__ losses) {
    losses[(step[1] - 1) % spe] = src[0];
}

unsigned blocks(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

struct orkan_mlp {
    int n_in = 0, h = 0, maxb = 0;
    size_t np = 0;
    // parameter-vector offsets
    size_t oW1, ob1, oW2, ob2, oW3, ob3;
    float *P = nullptr, *G = nullptr, *M1 = nullptr, *M2 = nullptr;
    float *Z1 = nullptr, *A1 = nullptr, *Z2 = nullptr, *A2 = nullptr, *y = nullptr, *dy = nullptr;
    float *dZ2 = nullptr, *dZ1 = nullptr, *xb = nullptr, *tb = nullptr, *loss = nullptr, *losses = nullptr;
    float* split = nullptr;             // k-slice partial products of the weight gradients
    size_t split_cap = 0;
    unsigned* step = nullptr;
    size_t losses_cap = 0;
};

namespace {

template <bool TA, bool TB, int EPI>
void gemm(cudaStream_t st, int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
          const float* bias = nullptr, const float* aux = nullptr, float* out2 = nullptr) {
    const dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM);
    if (grid.x * grid.y >= 148) {
        k_gemm<TA, TB, EPI><<<grid, kGemmThreads, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, aux, out2);
    } else {                                   // 32 x 32 tiles: four times the blocks
        const dim3 g2((N + 31) / 32, (M + 31) / 32);
        k_gemm<TA, TB, EPI, 32, 32><<<g2, kGemmThreads, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, aux, out2);
    }
    ++g_launches;
}

// C[M][N] (ldc = N) = sum over a long k (the batch) of A^T B, split into k slices so that
// the grid covers the SMs; the slices are summed in order (deterministic).
void gemm_tn_split(orkan_mlp* m, cudaStream_t st, int M, int N, int K, const float* A, int lda, const float* B,
                   int ldb, float* C) {
    const int tiles = ((N + kBN - 1) / kBN) * ((M + kBM - 1) / kBM);
    int nz = (296 + tiles - 1) / tiles;
    nz = std::max(1, std::min(nz, (K + kBK - 1) / kBK));
    if (nz == 1 || (size_t)nz * M * N > m->split_cap) {
        gemm<true, false, kEpiStore>(st, M, N, K, A, lda, B, ldb, C, N);
        return;
    }
    const dim3 grid((N + kBN - 1) / kBN, (M + kBM - 1) / kBM, nz);
    k_gemm<true, false, kEpiStore><<<grid, kGemmThreads, 0, st>>>(M, N, K, A, lda, B, ldb, m->split, N, nullptr,
                                                                  nullptr, nullptr);
    const size_t cnt = (size_t)M * N;
    k_sum_slices<<<blocks(cnt, 256), 256, 0, st>>>(m->split, nz, cnt, C);
    g_launches += 2;
}

// Forward of `batch` rows of x into m->Z1, A1, Z2, A2, y.
void forward(orkan_mlp* m, const float* x, int batch, float* y, cudaStream_t st) {
    const int I = m->n_in, H = m->h;
    gemm<false, false, kEpiBiasGelu>(st, batch, H, I, x, I, m->P + m->oW1, H, m->Z1, H, m->P + m->ob1, nullptr, m->A1);
    gemm<false, false, kEpiBiasGelu>(st, batch, H, H, m->A1, H, m->P + m->oW2, H, m->Z2, H, m->P + m->ob2, nullptr,
                                     m->A2);
    k_rowdot<<<blocks(batch, 8), 256, 0, st>>>(m->A2, batch, H, m->P + m->oW3, m->P + m->ob3, y);
    ++g_launches;
}

// Backward from dy (m->dy) into the gradient vector g and, optionally, dL/dx.
void backward(orkan_mlp* m, const float* x, int batch, float* g, float* gx, cudaStream_t st) {
    const int I = m->n_in, H = m->h;
    k_coldot<<<blocks(H, 128), 128, 0, st>>>(m->A2, batch, H, m->dy, g + m->oW3);
    k_colsum<<<1, 32, 0, st>>>(m->dy, batch, 1, g + m->ob3);
    k_outer_gelu<<<blocks((size_t)batch * H, 256), 256, 0, st>>>(m->dy, m->P + m->oW3, m->Z2, batch, H, m->dZ2);
    g_launches += 3;
    gemm_tn_split(m, st, H, H, batch, m->A1, H, m->dZ2, H, g + m->oW2);
    k_colsum<<<blocks(H, 128), 128, 0, st>>>(m->dZ2, batch, H, g + m->ob2);
    ++g_launches;
    gemm<false, true, kEpiGeluBack>(st, batch, H, H, m->dZ2, H, m->P + m->oW2, H, m->dZ1, H, nullptr, m->Z1);
    gemm_tn_split(m, st, I, H, batch, x, I, m->dZ1, H, g + m->oW1);
    k_colsum<<<blocks(H, 128), 128, 0, st>>>(m->dZ1, batch, H, g + m->ob1);
    ++g_launches;
    if (gx) gemm<false, true, kEpiStore>(st, batch, I, H, m->dZ1, H, m->P + m->oW1, H, gx, I);
}

// One training step on the minibatch of the device step counter (captured into a graph).
void train_step(orkan_mlp* m, const float* X, const float* T, unsigned count, int batch, unsigned spe, uint64_t seed,
                float lr, cudaStream_t st) {
    k_step_begin<<<1, 1, 0, st>>>(m->step);
    k_gather<<<blocks(batch, 128), 128, 0, st>>>(X, T, count, m->n_in, batch, spe, seed, m->step, m->xb, m->tb);
    g_launches += 2;
    forward(m, m->xb, batch, m->y, st);
    k_loss<<<1, 1024, 0, st>>>(m->y, m->tb, batch, m->dy, m->loss);
    k_copy_loss<<<1, 1, 0, st>>>(m->loss, m->step, spe, m->losses);
    g_launches += 2;
    backward(m, m->xb, batch, m->G, nullptr, st);
    k_adam<<<blocks(m->np, 256), 256, 0, st>>>(m->P, m->G, m->M1, m->M2, m->np, lr, m->step);
    ++g_launches;
}

}  // namespace

extern "C" {

int orkan_mlp_create(orkan_mlp_t** out, unsigned n_in, unsigned hidden, unsigned max_batch, unsigned long long seed) {
    if (!out) return (int)cudaErrorInvalidValue;
    *out = nullptr;
    if (n_in == 0 || hidden == 0 || max_batch == 0 || n_in > 4096 || hidden > 8192 || max_batch > (1u << 22))
        return (int)cudaErrorInvalidValue;
    orkan_mlp* m = new orkan_mlp();
    m->n_in = (int)n_in;
    m->h = (int)hidden;
    m->maxb = (int)max_batch;
    const size_t I = n_in, H = hidden, B = max_batch;
    m->oW1 = 0;
    m->ob1 = m->oW1 + I * H;
    m->oW2 = m->ob1 + H;
    m->ob2 = m->oW2 + H * H;
    m->oW3 = m->ob2 + H;
    m->ob3 = m->oW3 + H;
    m->np = m->ob3 + 1;
    int rc = 0;
    auto al = [&](float** p, size_t n) {
        if (!rc) rc = (int)cudaMalloc(reinterpret_cast<void**>(p), (n ? n : 1) * sizeof(float));
    };
    al(&m->P, m->np);
    al(&m->G, m->np);
    al(&m->M1, m->np);
    al(&m->M2, m->np);
    al(&m->Z1, B * H);
    al(&m->A1, B * H);
    al(&m->Z2, B * H);
    al(&m->A2, B * H);
    al(&m->dZ2, B * H);
    al(&m->dZ1, B * H);
    al(&m->y, B);
    al(&m->dy, B);
    al(&m->xb, B * I);
    al(&m->tb, B);
    al(&m->loss, 1);
    m->split_cap = (size_t)32 * std::max(I, H) * H;
    al(&m->split, m->split_cap);
    if (!rc) rc = (int)cudaMalloc(reinterpret_cast<void**>(&m->step), 2 * sizeof(unsigned));
    if (rc) {
        orkan_mlp_destroy(m);
        return rc;
    }
    // deterministic initialisation: splitmix64 stream, uniform in +-sqrt(6 / fan_in) for W
    std::vector<float> p(m->np, 0.0f);
    uint64_t st = seed;
    auto uni = [&](float bound) {
        st += 0x9e3779b97f4a7c15ull;
        const uint64_t z = mix64(st);
        return (float)(((double)(z >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0) * bound;
    };
    const float b1 = sqrtf(6.0f / (float)I), b2 = sqrtf(6.0f / (float)H);
    for (size_t i = 0; i < I * H; ++i) p[m->oW1 + i] = uni(b1);
    for (size_t i = 0; i < H * H; ++i) p[m->oW2 + i] = uni(b2);
    for (size_t i = 0; i < H; ++i) p[m->oW3 + i] = uni(b2);
    rc = orkan_mlp_set_params(m, p.data());
    if (rc) {
        orkan_mlp_destroy(m);
        return rc;
    }
    *out = m;
    return 0;
}

void orkan_mlp_destroy(orkan_mlp_t* m) {
    if (!m) return;
    float* bufs[] = {m->P, m->G, m->M1, m->M2, m->Z1, m->A1, m->Z2, m->A2, m->dZ2, m->dZ1,
                     m->y, m->dy, m->xb, m->tb, m->loss, m->losses, m->split};
    for (float* b : bufs) cudaFree(b);
    cudaFree(m->step);
    delete m;
}

size_t orkan_mlp_param_count(const orkan_mlp_t* m) { return m ? m->np : 0; }

int orkan_mlp_get_params(const orkan_mlp_t* m, float* host) {
    if (!m || !host) return (int)cudaErrorInvalidValue;
    return (int)cudaMemcpy(host, m->P, m->np * sizeof(float), cudaMemcpyDeviceToHost);
}

int orkan_mlp_set_params(orkan_mlp_t* m, const float* host) {
    if (!m || !host) return (int)cudaErrorInvalidValue;
    int rc = (int)cudaMemcpy(m->P, host, m->np * sizeof(float), cudaMemcpyHostToDevice);
    if (!rc) rc = (int)cudaMemset(m->M1, 0, m->np * sizeof(float));
    if (!rc) rc = (int)cudaMemset(m->M2, 0, m->np * sizeof(float));
    if (!rc) rc = (int)cudaMemset(m->step, 0, 2 * sizeof(unsigned));
    return rc;
}

int orkan_mlp_forward(orkan_mlp_t* m, const float* x_dev, unsigned batch, float* y_dev, void* stream) {
    if (!m || !x_dev || !y_dev || batch == 0 || (int)batch > m->maxb) return (int)cudaErrorInvalidValue;
    forward(m, x_dev, (int)batch, y_dev, reinterpret_cast<cudaStream_t>(stream));
    return (int)cudaGetLastError();
}

int orkan_mlp_gradients(orkan_mlp_t* m, const float* x_dev, const float* t_dev, unsigned batch, float* loss_dev,
                        float* grad_dev, float* gx_dev, void* stream) {
    if (!m || !x_dev || !t_dev || !grad_dev || batch == 0 || (int)batch > m->maxb) return (int)cudaErrorInvalidValue;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    forward(m, x_dev, (int)batch, m->y, st);
    k_loss<<<1, 1024, 0, st>>>(m->y, t_dev, (int)batch, m->dy, loss_dev);
    ++g_launches;
    backward(m, x_dev, (int)batch, grad_dev, gx_dev, st);
    return (int)cudaGetLastError();
}

int orkan_mlp_train(orkan_mlp_t* m, const float* x_dev, const float* t_dev, unsigned count, unsigned epochs,
                    unsigned batch, float lr, unsigned long long seed, float* loss_dev, void* stream) {
    if (!m || !x_dev || !t_dev || batch == 0 || (int)batch > m->maxb || count < batch)
        return (int)cudaErrorInvalidValue;
    if (epochs == 0) return 0;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const unsigned spe = count / batch;
    int rc = 0;
    if (spe > m->losses_cap) {
        cudaFree(m->losses);
        m->losses = nullptr;
        m->losses_cap = 0;
        if ((rc = (int)cudaMalloc(reinterpret_cast<void**>(&m->losses), spe * sizeof(float)))) return rc;
        m->losses_cap = spe;
    }
    // step[0] counts every Adam step of this network (bias correction); step[1] restarts at
    // 0 for this call and drives the epoch schedule
    if ((rc = (int)cudaMemsetAsync(m->step + 1, 0, sizeof(unsigned), st))) return rc;
    cudaStream_t cap = nullptr;
    if ((rc = (int)cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking))) return rc;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    const unsigned long long l0 = g_launches.load();
    rc = (int)cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (!rc) {
        train_step(m, x_dev, t_dev, count, (int)batch, spe, seed, lr, cap);
        const int erc = (int)cudaGetLastError();
        rc = (int)cudaStreamEndCapture(cap, &g);
        if (!rc) rc = erc;
    }
    const unsigned long long per_step = g_launches.load() - l0;
    g_launches -= per_step;                       // counted per replay below
    if (!rc) rc = (int)cudaGraphInstantiate(&ge, g, 0);
    if (g) cudaGraphDestroy(g);
    cudaEvent_t ev = nullptr;                     // the replays follow the caller's stream
    if (!rc) rc = (int)cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (!rc) rc = (int)cudaEventRecord(ev, st);
    if (!rc) rc = (int)cudaStreamWaitEvent(cap, ev, 0);
    const unsigned long long total = (unsigned long long)epochs * spe;
    for (unsigned long long s = 0; s < total && !rc; ++s) {
        rc = (int)cudaGraphLaunch(ge, cap);
        g_launches += per_step;
    }
    if (!rc && loss_dev) {
        k_epoch_loss<<<1, 1, 0, cap>>>(m->losses, spe, loss_dev);
        ++g_launches;
        rc = (int)cudaGetLastError();
    }
    if (!rc) rc = (int)cudaEventRecord(ev, cap);
    if (!rc) rc = (int)cudaStreamWaitEvent(st, ev, 0);
    if (!rc) rc = (int)cudaStreamSynchronize(cap);
    if (ge) cudaGraphExecDestroy(ge);
    if (ev) cudaEventDestroy(ev);
    cudaStreamDestroy(cap);
    return rc;
}

int orkan_mlp_ascend(orkan_mlp_t* m, float* x_dev, unsigned count, unsigned steps, float lr, float lo, float hi,
                     float* y_dev, void* stream) {
    if (!m || !x_dev || count == 0) return (int)cudaErrorInvalidValue;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const size_t nx = (size_t)count * m->n_in;
    float *gx = nullptr, *m1 = nullptr, *m2 = nullptr;
    int rc = 0;
    if ((rc = (int)cudaMalloc(reinterpret_cast<void**>(&gx), nx * sizeof(float))) ||
        (rc = (int)cudaMalloc(reinterpret_cast<void**>(&m1), nx * sizeof(float))) ||
        (rc = (int)cudaMalloc(reinterpret_cast<void**>(&m2), nx * sizeof(float)))) {
        cudaFree(gx);
        cudaFree(m1);
        return rc;
    }
    cudaMemsetAsync(m1, 0, nx * sizeof(float), st);
    cudaMemsetAsync(m2, 0, nx * sizeof(float), st);
    for (unsigned t = 1; t <= steps && !rc; ++t) {
        for (unsigned c0 = 0; c0 < count; c0 += (unsigned)m->maxb) {
            const int b = (int)((count - c0) < (unsigned)m->maxb ? count - c0 : (unsigned)m->maxb);
            const float* xc = x_dev + (size_t)c0 * m->n_in;
            forward(m, xc, b, m->y, st);
            k_loss<<<1, 1024, 0, st>>>(m->y, nullptr, b, m->dy, nullptr);
            ++g_launches;
            backward(m, xc, b, m->G, gx + (size_t)c0 * m->n_in, st);
        }
        k_adam_inputs<<<blocks(nx, 256), 256, 0, st>>>(x_dev, gx, m1, m2, nx, lr, (int)t, lo, hi);
        ++g_launches;
        rc = (int)cudaGetLastError();
    }
    if (!rc && y_dev) {
        for (unsigned c0 = 0; c0 < count; c0 += (unsigned)m->maxb) {
            const int b = (int)((count - c0) < (unsigned)m->maxb ? count - c0 : (unsigned)m->maxb);
            forward(m, x_dev + (size_t)c0 * m->n_in, b, y_dev + c0, st);
        }
        rc = (int)cudaGetLastError();
    }
    if (!rc) rc = (int)cudaStreamSynchronize(st);
    cudaFree(gx);
    cudaFree(m1);
    cudaFree(m2);
    return rc;
}

unsigned long long orkan_mlp_launch_count(void) { return g_launches.load(); }

}  // extern "C"
