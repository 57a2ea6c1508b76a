/*
 * runtime.c - library stream, device allocation, staging of caller arrays, error
 * reporting, and the orkan_dev.h extensions.
 */
#include "internal.h"

#include <cuda_runtime_api.h>
#include <pthread.h>
#include <string.h>

extern void *orkan_internal_staging(size_t bytes);   /* csrc/cuda/scratch.cu */

static void *g_stream = NULL;
static int g_fail_allocs = 0;

int orkan_log_tile_dim(void) { return LOG_TILE_DIM; }
void orkan_set_stream(void *stream) {
    orkan_flush();                              /* queued gates go to the old stream */
    g_stream = stream;
}
void *orkan_get_stream(void) { return g_stream; }
void *orkan_stream(void) { return g_stream; }
unsigned long long orkan_launch_count(void) { return orkan_cu_launch_count(); }
void orkan_debug_fail_allocs(int n) { g_fail_allocs = n > 0 ? n : 0; }

void orkan_sync(void) {
    orkan_flush();
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

/* ---- cache of host arrays staged to the device ---------------------------------------
 * Off by default (every call copies the host array, so a caller may change it between
 * calls).  orkan_set_host_array_cache(bytes) keeps up to that many bytes of staged arrays
 * on the device, keyed by host pointer, length and a generation counter: a call with the
 * same pointer and length in the same generation reuses the device copy.  A caller that
 * changes a cached array in place calls orkan_host_arrays_changed() (a new generation)
 * before its next call.  The least recently used entries are freed to make room. */
#define HCACHE_SLOTS 8
static pthread_mutex_t g_hc_mu = PTHREAD_MUTEX_INITIALIZER;
static size_t g_hc_budget = 0;
static unsigned long long g_hc_gen = 1, g_hc_tick = 0, g_hc_hits = 0, g_hc_misses = 0;
static struct {
    const void *host;
    size_t n;
    unsigned long long gen, used;
    int dev;
    double *buf;
} g_hc[HCACHE_SLOTS];

static void hc_free_slot(int i) {
    if (g_hc[i].buf) cudaFree(g_hc[i].buf);
    memset(&g_hc[i], 0, sizeof(g_hc[i]));
}

void orkan_set_host_array_cache(size_t max_bytes) {
    pthread_mutex_lock(&g_hc_mu);
    g_hc_budget = max_bytes;
    for (int i = 0; i < HCACHE_SLOTS; ++i)
        if (g_hc[i].buf) hc_free_slot(i);
    pthread_mutex_unlock(&g_hc_mu);
}

void orkan_host_arrays_changed(void) {
    pthread_mutex_lock(&g_hc_mu);
    ++g_hc_gen;
    pthread_mutex_unlock(&g_hc_mu);
}

void orkan_host_array_cache_stats(unsigned long long *hits, unsigned long long *misses) {
    pthread_mutex_lock(&g_hc_mu);
    if (hits) *hits = g_hc_hits;
    if (misses) *misses = g_hc_misses;
    pthread_mutex_unlock(&g_hc_mu);
}

/* The cached device copy of host array p (n doubles), staging it on a miss; NULL when the
 * cache is off or the array does not fit its budget. */
static const double *hc_lookup(const char *module, const double *p, size_t n) {
    const size_t bytes = n * sizeof(double);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return NULL;
    }
    pthread_mutex_lock(&g_hc_mu);
    if (bytes == 0 || bytes > g_hc_budget) {
        pthread_mutex_unlock(&g_hc_mu);
        return NULL;
    }
    for (int i = 0; i < HCACHE_SLOTS; ++i)
        if (g_hc[i].buf && g_hc[i].host == p && g_hc[i].n == n && g_hc[i].dev == dev && g_hc[i].gen == g_hc_gen) {
            g_hc[i].used = ++g_hc_tick;
            ++g_hc_hits;
            double *hit = g_hc[i].buf;
            pthread_mutex_unlock(&g_hc_mu);
            return hit;
        }
    /* make room: stale entries first, then the least recently used */
    for (int i = 0; i < HCACHE_SLOTS; ++i)
        if (g_hc[i].buf && (g_hc[i].gen != g_hc_gen || (g_hc[i].host == p && g_hc[i].dev == dev))) hc_free_slot(i);
    for (;;) {
        size_t held = 0;
        int free_slot = -1, lru = -1;
        for (int i = 0; i < HCACHE_SLOTS; ++i) {
            if (!g_hc[i].buf) { if (free_slot < 0) free_slot = i; continue; }
            held += g_hc[i].n * sizeof(double);
            if (lru < 0 || g_hc[i].used < g_hc[lru].used) lru = i;
        }
        if (free_slot >= 0 && held + bytes <= g_hc_budget) {
            double *buf = NULL;
            if (cudaMalloc((void **)&buf, bytes) != cudaSuccess) {
                cudaGetLastError();
                pthread_mutex_unlock(&g_hc_mu);
                return NULL;
            }
            cudaError_t e = cudaMemcpyAsync(buf, p, bytes, cudaMemcpyHostToDevice, (cudaStream_t)g_stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)g_stream);
            if (e != cudaSuccess) {
                cudaFree(buf);
                pthread_mutex_unlock(&g_hc_mu);
                orkan_check_cu(module, "copy of a host array to the device", (int)e);
            }
            g_hc[free_slot].host = p;
            g_hc[free_slot].n = n;
            g_hc[free_slot].gen = g_hc_gen;
            g_hc[free_slot].used = ++g_hc_tick;
            g_hc[free_slot].dev = dev;
            g_hc[free_slot].buf = buf;
            ++g_hc_misses;
            pthread_mutex_unlock(&g_hc_mu);
            return buf;
        }
        if (lru < 0) break;
        hc_free_slot(lru);
    }
    pthread_mutex_unlock(&g_hc_mu);
    return NULL;
}

const double *orkan_device_doubles(const char *module, const double *p, size_t n) {
    if (is_device_pointer(p)) return p;
    const double *cached = hc_lookup(module, p, n);
    if (cached) return cached;
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
    orkan_flush();
    const size_t bytes = (size_t)state_len(state) * sizeof(cplx_t);
    cudaError_t e = cudaMemcpyAsync(state->data, host, bytes, cudaMemcpyHostToDevice, (cudaStream_t)g_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)g_stream);
    return (int)e;
}

int orkan_state_upload_async(state_t *state, const cplx_t *host, void *stream) {
    if (!state || !state->data || !host) return (int)cudaErrorInvalidValue;
    orkan_flush();
    const size_t bytes = (size_t)state_len(state) * sizeof(cplx_t);
    cudaStream_t st = stream ? (cudaStream_t)stream : (cudaStream_t)g_stream;
    cudaError_t e = cudaSuccess;
    if (st != (cudaStream_t)g_stream) {
        /* the copy waits for the library stream's work enqueued so far */
        cudaEvent_t ev;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return (int)e;
        e = cudaEventRecord(ev, (cudaStream_t)g_stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ev, 0);
        cudaEventDestroy(ev);
        if (e != cudaSuccess) return (int)e;
    }
    return (int)cudaMemcpyAsync(state->data, host, bytes, cudaMemcpyHostToDevice, st);
}

int orkan_state_download(const state_t *state, cplx_t *host) {
    if (!state || !state->data || !host) return (int)cudaErrorInvalidValue;
    orkan_flush();
    const size_t bytes = (size_t)state_len(state) * sizeof(cplx_t);
    cudaError_t e = cudaMemcpyAsync(host, state->data, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)g_stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)g_stream);
    return (int)e;
}
