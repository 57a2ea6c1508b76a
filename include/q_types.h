/*
 * q_types.h - scalar types and tile geometry shared by every Orkan-B200 header.
 *
 * ABI-identical to the reference's include/q_types.h:29-57 (same typedefs, same
 * enum values, same macros), so code compiled against the reference headers links
 * against this library unchanged.  The state buffers these types describe live in
 * GPU memory in this build; see state.h.
 */
#ifndef QTYPES_H
#define QTYPES_H

#include <stdint.h>
#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes (reference include/q_types.h:29-38).  Declared for ABI parity;
 * like the reference, the public calls report errors by message + exit(). */
typedef enum {
    QS_OK           =  0,
    QS_ERR_NULL     = -1,
    QS_ERR_OOM      = -2,
    QS_ERR_QUBIT    = -3,
    QS_ERR_TYPE     = -4,
    QS_ERR_FILE     = -5,
    QS_ERR_FORMAT   = -6,
    QS_ERR_PARAM    = -7,
} qs_error_t;

typedef unsigned char   qubit_t;   /* qubit index                                   */
typedef double _Complex cplx_t;    /* one amplitude / matrix element, 16 bytes       */
typedef uint64_t        idx_t;     /* storage index; dim^2 exceeds 32 bits at 16 q  */

/* Tile geometry of the MIXED_TILED layout.  LOG_TILE_DIM is part of the ABI: the
 * library and its callers must agree on it (the reference passes it as a PUBLIC
 * CMake definition, src/CMakeLists.txt:101-104).  liborkan_b200.so is built with
 * 5 (32x32 tiles, the reference Release value); liborkan_b200_t3.so with 3
 * (8x8 tiles, the reference Debug value).  orkan_log_tile_dim() in orkan_dev.h
 * returns the value a loaded library was built with. */
#ifndef LOG_TILE_DIM
#define LOG_TILE_DIM 5
#endif
#define TILE_DIM  (1 << LOG_TILE_DIM)
#define TILE_SIZE (TILE_DIM * TILE_DIM)

#ifndef MIN
    #define MIN(a,b)                ((a) < (b) ? (a) : (b))
#endif
#ifndef MAX
    #define MAX(a,b)                ((a) > (b) ? (a) : (b))
#endif
#define SWAP(a, b, T)           do { T q; q = *(a); *(a) = *(b); *(b) = q; } while(0)
#define POW2(a, T)              (((T)1) << (a))

#ifdef __cplusplus
}
#endif

#endif /* QTYPES_H */
