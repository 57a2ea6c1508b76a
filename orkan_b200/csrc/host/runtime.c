/*
 * runtime.c - library stream, device allocation, staging of caller arrays, error
 * reporting, and the orkan_dev.h extensions.
 */
#include "internal.h"

#include <cuda_runtime_api.h>
#include <string.h>

extern void *orkan_internal_staging(size_t bytes);   /* csrc/cuda/scratch.cu */

static void *g_stream = NULL;
static int g_fail_allocs = 0;

int orkan_log_tile_dim(void) { return LOG_TILE_DIM; }
void orkan_set_stream(void *stream) { g_stream = stream; }
void *orkan_get_stream(void) { return g_stream; }
void *orkan_stream(void) { return g_stream; }
unsigned long long orkan_launch_count(void) { return orkan_cu_launch_count(); }
void orkan_debug_fail_allocs(int n) { g_fail_allocs = n > 0 ? n : 0; }

void orkan_sync(void) {
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)g_stream);
    if (e != cudaSuccess) {
        fprintf(stderr, "orkan: runtime: stream synchronisation failed: %s\n", cudaGetErrorString(e));
        exit(EXIT_FAILURE);
    }
}

void orkan_check_cu(const char *module, const char *what, int rc) {
    if (rc == 0) return;
    fprintf(stderr, "orkan: %s: %s: CUDA error %d (%s)\n", module, what, rc,
            cudaGetErrorString((cudaError_t)rc));
    exit(EXIT_FAILURE);
}

cplx_t *orkan_alloc_state(idx_t len) {
    if (g_fail_allocs > 0) {
        --g_fail_allocs;
        return NULL;
    }
    void *p = NULL;
    const size_t bytes = (size_t)len * sizeof(cplx_t);
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
        cudaGetLastError();
        return NULL;
    }
    if (cudaMemsetAsync(p, 0, bytes, (cudaStream_t)g_stream) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
        return NULL;
    }
    return (cplx_t *)p;
}

void orkan_free_device(void *p) {
    if (p) cudaFree(p);
}

/* Is p device-accessible memory the kernels can read directly? */
static int is_device_pointer(const void *p) {
    struct cudaPointerAttributes a;
    memset(&a, 0, sizeof(a));
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static int is_pinned_host_pointer(const void *p) {
    struct cudaPointerAttributes a;
    memset(&a, 0, sizeof(a));
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeHost;
}

const double *orkan_device_doubles(const char *module, const double *p, size_t n) {
    if (is_device_pointer(p)) return p;
    double *buf = (double *)orkan_internal_staging(n * sizeof(double));
    if (!buf) {
        fprintf(stderr, "orkan: %s: cannot allocate the device staging buffer\n", module);
        exit(EXIT_FAILURE);
    }
    cudaError_t e = cudaMemcpyAsync(buf, p, n * sizeof(double), cudaMemcpyHostToDevice, (cudaStream_t)g_stream);
    /* a pinned source is read asynchronously: wait so the caller may reuse it on return */
    if (e == cudaSuccess && is_pinned_host_pointer(p)) e = cudaStreamSynchronize((cudaStream_t)g_stream);
    orkan_check_cu(module, "copy of a host array to the device", (int)e);
    return buf;
}

int orkan_state_upload(state_t *state, const cplx_t *host) {
    if (!state || !state->data || !host) return (int)cudaErrorInvalidValue;
    const size_t bytes = (size_t)state_len(state) * sizeof(cplx_t);
    cudaError_t e = cudaMemcpyAsync(state->data, host, bytes, cudaMemcpyHostToDevice, (cudaStream_t)g_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)g_stream);
    return (int)e;
}

int orkan_state_download(const state_t *state, cplx_t *host) {
    if (!state || !state->data || !host) return (int)cudaErrorInvalidValue;
    const size_t bytes = (size_t)state_len(state) * sizeof(cplx_t);
    cudaError_t e = cudaMemcpyAsync(host, state->data, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)g_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)g_stream);
    return (int)e;
}
