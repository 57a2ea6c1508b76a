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


def _declare(lib):
    lib.orkan_cu_exp_diag_noalloc.argtypes = [C.c_int, C.c_uint, C.c_void_p, C.c_uint, C.c_void_p, C.c_double,
                                              C.c_void_p]
    lib.orkan_cu_exp_diag_noalloc.restype = C.c_int
    lib.orkan_cu_exp_diag.argtypes = lib.orkan_cu_exp_diag_noalloc.argtypes
    lib.orkan_cu_exp_diag.restype = C.c_int


def test_noalloc_full_table_at_16_qubits_against_oracle(ork5):
    """16 qubits use all 65536 table entries.  The tiled density matrix (34 GB) is compared
    with the regular path over its whole storage on the device, and a 48 x 48 block of rows
    and columns that includes the last indices is compared with the oracle."""
    import torch
    from orkan_b200 import workloads as W
    _declare(ork5.lib)
    n, d, t = 16, 1 << 16, 0.83
    rng = np.random.default_rng(16)
    diag_h = rng.uniform(-3, 3, d)
    diag = torch.from_numpy(diag_h).cuda()
    a, b = ork5.plus("tiled", n), ork5.plus("tiled", n)
    for _ in range(2):                                   # two calls in a row on the shared table
        assert ork5.lib.orkan_cu_exp_diag(2, 5, a.data, n, diag.data_ptr(), t, None) == 0
        assert ork5.lib.orkan_cu_exp_diag_noalloc(2, 5, b.data, n, diag.data_ptr(), t, None) == 0
        torch.cuda.synchronize()
        va, vb = W.state_view(ork5, a), W.state_view(ork5, b)
        assert float((va - vb).abs().max()) <= TOL
        del va, vb
    rows = np.unique(np.concatenate([[0, 1, 31, 32, d - 33, d - 32, d - 2, d - 1], rng.integers(0, d, 40)]))
    sub = np.full((len(rows), len(rows)), 1.0 / d, dtype=np.complex128)
    want = R.exp_diag("packed", R.exp_diag("packed", sub, diag_h[rows], t), diag_h[rows], t)
    err = max(abs(ork5.get(b, int(r), int(c)) - want[i, j])
              for i, r in enumerate(rows) for j, c in enumerate(rows) if r >= c)
    assert err <= TOL
    ork5.free(a)
    ork5.free(b)


def test_noalloc_t_zero_leaves_the_state_bit_identical(ork5):
    import torch
    _declare(ork5.lib)
    for kind, layout in (("packed", 1), ("tiled", 2)):
        start = R.to_storage(kind, _rand_rho(6, 9), 5)
        st = ork5.state(kind, 6, start)
        diag = torch.linspace(-1, 1, 64, dtype=torch.float64, device="cuda")
        assert ork5.lib.orkan_cu_exp_diag_noalloc(layout, 5, st.data, 6, diag.data_ptr(), 0.0, None) == 0
        torch.cuda.synchronize()
        assert np.array_equal(ork5.storage(st), start)
        ork5.free(st)


def test_noalloc_rejects_sizes_beyond_its_table(ork5):
    _declare(ork5.lib)
    st = ork5.state("packed", 2)
    diag = np.zeros(4)
    # 17 qubits exceed the 65536-entry table: rejected before any launch or memory access
    assert ork5.lib.orkan_cu_exp_diag_noalloc(1, 5, st.data, 17, diag.ctypes.data, 0.5, None) != 0
    # tile geometries outside 1..8 and layouts other than packed/tiled are rejected too
    assert ork5.lib.orkan_cu_exp_diag_noalloc(2, 0, st.data, 2, diag.ctypes.data, 0.5, None) != 0
    assert ork5.lib.orkan_cu_exp_diag_noalloc(2, 9, st.data, 2, diag.ctypes.data, 0.5, None) != 0
    assert ork5.lib.orkan_cu_exp_diag_noalloc(0, 5, st.data, 2, diag.ctypes.data, 0.5, None) != 0
    ork5.free(st)
