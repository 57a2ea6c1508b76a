"""The allocation-free exp_diag entry point (orkan_cu_exp_diag_noalloc), called through
the C ABI, against the existing orkan_cu_exp_diag on identical inputs.

It serves callers that cannot let the library allocate device memory: programs whose own
pool allocator already holds nearly all of it, and latency-sensitive callers that cannot
absorb the device-wide wait of cudaFree when the regular path grows its scratch buffer.
Its phase table is a fixed device array shared by all calls, so the test makes two calls
in a row (different diagonal, different t, different layout) and checks both.  This file
is collected last so that a run stopping at its first failure has run everything else."""
import ctypes as C

import numpy as np
import pytest

from oracle import restate as R

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _rand_rho(n, seed):
    rng = np.random.default_rng(seed)
    d = 1 << n
    a = rng.standard_normal((d, 3)) + 1j * rng.standard_normal((d, 3))
    rho = a @ a.conj().T
    return rho / np.trace(rho).real


def test_noalloc_exp_diag_matches_regular_path_twice(ork5):
    import torch
    lib = ork5.lib
    lib.orkan_cu_exp_diag_noalloc.argtypes = [C.c_int, C.c_uint, C.c_void_p, C.c_uint, C.c_void_p, C.c_double,
                                              C.c_void_p]
    lib.orkan_cu_exp_diag_noalloc.restype = C.c_int
    lib.orkan_cu_exp_diag.argtypes = lib.orkan_cu_exp_diag_noalloc.argtypes
    lib.orkan_cu_exp_diag.restype = C.c_int
    calls = [("packed", 1, 10, 0.61, 1), ("tiled", 2, 9, -1.37, 2)]
    for kind, layout, n, t, seed in calls:
        start = R.to_storage(kind, _rand_rho(n, seed), 5)
        a, b = ork5.state(kind, n, start), ork5.state(kind, n, start)
        diag = torch.tensor(np.random.default_rng(seed).uniform(-4, 4, 1 << n), dtype=torch.float64, device="cuda")
        rc1 = lib.orkan_cu_exp_diag(layout, 5, a.data, n, diag.data_ptr(), t, None)
        rc2 = lib.orkan_cu_exp_diag_noalloc(layout, 5, b.data, n, diag.data_ptr(), t, None)
        torch.cuda.synchronize()
        assert rc1 == 0 and rc2 == 0
        regular, noalloc = ork5.storage(a), ork5.storage(b)
        assert np.abs(noalloc - regular).max() <= TOL
        assert np.abs(noalloc - start).max() > 1e-3          # the call did change the state
        ork5.free(a)
        ork5.free(b)


def test_noalloc_rejects_sizes_beyond_its_table(ork5):
    lib = ork5.lib
    lib.orkan_cu_exp_diag_noalloc.argtypes = [C.c_int, C.c_uint, C.c_void_p, C.c_uint, C.c_void_p, C.c_double,
                                              C.c_void_p]
    lib.orkan_cu_exp_diag_noalloc.restype = C.c_int
    st = ork5.state("packed", 2)
    diag = np.zeros(4)
    # 17 qubits exceed the 65536-entry table: rejected before any launch or memory access
    assert lib.orkan_cu_exp_diag_noalloc(1, 5, st.data, 17, diag.ctypes.data, 0.5, None) != 0
    ork5.free(st)
