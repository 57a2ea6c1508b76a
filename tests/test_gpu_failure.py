"""Failure detection of the density-matrix engine, driven without a GPU fault.

Every wait of the engine for its staged data is bounded; a wait that runs out sets bit 0
of a device error word (orkan_cu_engine_status) and the kernel returns instead of waiting
forever.  The test hook orkan_cu_engine_test_wait shortens the limit and arms each item's
completion barrier without issuing its copies, so the wait runs out with nothing in
flight.  The test checks that the launch ends promptly, that the host reads the error
status, that the word can be cleared, and that the context stays usable afterwards."""
import ctypes as C
import time

import numpy as np
import pytest

from oracle import restate as R

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _declare(lib):
    lib.orkan_cu_engine_status.restype = C.c_uint
    lib.orkan_cu_engine_status_clear.restype = C.c_int
    lib.orkan_cu_engine_test_wait.argtypes = [C.c_ulonglong, C.c_int]
    lib.orkan_cu_engine_test_wait.restype = None


@pytest.mark.parametrize("kind", ["tiled", "packed"])
def test_engine_wait_that_runs_out_reports_an_error(ork5, kind):
    lib = ork5.lib
    _declare(lib)
    assert lib.orkan_cu_engine_status_clear() == 0
    n = 7
    st = ork5.plus(kind, n)
    lib.orkan_cu_engine_test_wait(2048, 1)
    try:
        t0 = time.perf_counter()
        ork5.gate(st, "h", [3])
        ork5.sync()
        elapsed = time.perf_counter() - t0
    finally:
        lib.orkan_cu_engine_test_wait(0, 0)
    assert lib.orkan_cu_engine_status() & 1
    assert elapsed < 5.0
    assert lib.orkan_cu_engine_status_clear() == 0
    assert lib.orkan_cu_engine_status() == 0
    ork5.free(st)
    # the same gate on a fresh state now runs normally and matches the oracle
    st = ork5.plus(kind, n)
    ork5.gate(st, "h", [3])
    want = R.to_storage(kind, R.apply_gate(kind, R.plus_state(kind, n), "h", [3]), 5)
    err = np.abs(ork5.storage(st) - want).max()
    ork5.free(st)
    assert err <= TOL
    assert lib.orkan_cu_engine_status() == 0
