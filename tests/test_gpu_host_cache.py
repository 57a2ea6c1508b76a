"""The opt-in cache of host observable / diagonal arrays (orkan_set_host_array_cache,
include/orkan_dev.h): repeated calls with the same host array reuse its device copy; a
change made in place is seen only after orkan_host_arrays_changed(), as documented."""
import ctypes as C

import numpy as np
import pytest

from oracle import restate as R
from orkan_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _stats(lib):
    h, m = C.c_ulonglong(0), C.c_ulonglong(0)
    lib.orkan_host_array_cache_stats(C.byref(h), C.byref(m))
    return h.value, m.value


def test_host_array_cache(ork5):
    lib = ork5.lib
    lib.orkan_set_host_array_cache.argtypes = [C.c_size_t]
    lib.orkan_host_array_cache_stats.argtypes = [C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
    n = 10
    st = ork5.plus("pure", n)
    gates = W.random_circuit(n, 30, seed=4)
    psi = R.plus_state("pure", n)
    for g, qs, th in gates:
        ork5.gate(st, g, qs, th)
        psi = R.apply_pure(psi, g, qs, th)
    obs = np.random.default_rng(1).uniform(-1, 1, 1 << n)
    m0 = ork5.mean(st, obs)
    assert abs(m0 - R.mean("pure", psi, obs)) <= 1e-12
    lib.orkan_set_host_array_cache(1 << 20)
    try:
        h0, s0 = _stats(lib)
        m1, m2 = ork5.mean(st, obs), ork5.mean(st, obs)
        h1, s1 = _stats(lib)
        assert m1 == m0 and m2 == m0
        assert (h1 - h0, s1 - s0) == (1, 1)
        obs *= 2.0                                   # changed in place, not announced: stale copy
        assert ork5.mean(st, obs) == m0
        lib.orkan_host_arrays_changed()
        assert ork5.mean(st, obs) == 2.0 * m0
        # exp_diag reads its diagonal through the same cache
        ork5.exp_diag(st, obs, 0.3)
        psi = R.exp_diag("pure", psi, obs, 0.3)
        assert np.abs(ork5.storage(st) - psi).max() <= 1e-12
        # arrays above the budget are staged per call, not cached
        big = np.ones(1 << 18)
        h2, s2 = _stats(lib)
        st2 = ork5.plus("pure", 18)
        assert abs(ork5.mean(st2, big) - 1.0) <= 1e-12
        assert _stats(lib) == (h2, s2)
        ork5.free(st2)
    finally:
        lib.orkan_set_host_array_cache(0)
    ork5.free(st)
