/*
 * bench_blas_absent.c - the reference benchmark's BLAS rows where no CBLAS is installed.
 *
 * The reference's bench_main.c and bench_kraus_main.c register a dense-BLAS backend
 * (benchmark/src/bench_blas.c, bench_kraus_blas.c), which needs a CBLAS library.  This
 * machine has none, so these vtables report the backend unavailable at every size
 * (available() == 0), which the reference's drivers skip like a competitor that is not
 * built.
 */
#ifdef BENCH_B200_KRAUS
#include "bench_kraus.h"
#else
#include "bench.h"
#endif

static int absent_available(qubit_t q) { (void)q; return 0; }
static void absent_apply(void *ctx, const qubit_t *pos) { (void)ctx; (void)pos; }
static void absent_cleanup(void *ctx) { (void)ctx; }
static size_t absent_bytes(qubit_t q) { (void)q; return 0; }

#ifdef BENCH_B200_KRAUS
static void *absent_kraus_init(qubit_t q, int n_ops, int tgt, const cplx_t *ops) {
    (void)q; (void)n_ops; (void)tgt; (void)ops;
    return NULL;
}
const bench_kraus_backend_t kraus_blas_backend = {
    .name = "BLAS", .init = absent_kraus_init, .apply = absent_apply, .cleanup = absent_cleanup,
    .touch_bytes = absent_bytes, .available = absent_available
};
#else
static void *absent_init(qubit_t q, bench_gate_id_t g, double par) {
    (void)q; (void)g; (void)par;
    return NULL;
}
const bench_backend_t blas_backend = {
    .name = "BLAS", .init = absent_init, .apply = absent_apply, .cleanup = absent_cleanup,
    .touch_bytes = absent_bytes, .available = absent_available
};
#endif
