// scratch.cuh - per-device scratch buffers owned by the library.
//
// Slot 0 holds kernel scratch (reduction partials, exp_diag phase tables); slot 1 holds
// host arrays staged to the device (obs / diag passed as host pointers).  A buffer grows
// by freeing and reallocating; cudaFree waits for the device, so work still in flight
// on the old buffer completes first.  Calls from several host threads on one device are
// serialised by a mutex; concurrent use of one state from several threads is not
// supported (as in the reference).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace orkan {
void* scratch_get_slot(int slot, size_t bytes);
inline void* scratch_get(size_t bytes) { return scratch_get_slot(0, bytes); }
}  // namespace orkan
