"""The benchmark's algorithmic-byte model (orkan_b200/traffic.py) against brute-force
enumeration of the storage at small sizes (CPU only)."""
import itertools

import numpy as np
import pytest

from oracle import restate as R
from orkan_b200 import traffic as T
from orkan_b200 import workloads as W


def brute(kind, n, name, qs, lt):
    if kind == "pure":
        x = np.arange(1 << n)
        ch = T.pure_changes(name, qs)(x)
    else:
        if kind == "packed":
            r, c = R._packed_rc(n)
            live = np.ones(r.shape, dtype=bool)
        else:
            r, c, live = R._tiled_rc(n, lt)
        ch = T.mixed_changes(name, qs)(r, c) & live
    idx = np.nonzero(ch)[0]
    return len(np.unique(idx // 2))


@pytest.mark.parametrize("kind,lt", [("pure", 5), ("tiled", 3), ("tiled", 5), ("packed", 5)])
@pytest.mark.parametrize("n", [1, 2, 3, 5, 7])
def test_sector_counts_exact(kind, lt, n):
    for g in W.ALL_GATES + ("channel",):
        if kind == "pure" and g == "channel":
            continue
        k = 1 if g == "channel" else W.gate_arity(g)
        if k > n:
            continue
        for qs in itertools.permutations(range(n), k):
            got = T.sectors(kind, n, g, qs, lt)
            exp = brute(kind, n, g, qs, lt)
            assert got == exp, (g, qs, got, exp)


def test_dense_gates_equal_reference_convention():
    # 2 x storage bytes for gates that change every element (reference docs/BENCHMARK.md 6.2)
    for kind, n in (("pure", 20), ("tiled", 9), ("packed", 9)):
        length = R.state_len(kind, n, 5)
        assert T.gate_bytes(kind, n, "h", (3,)) == 2 * 32 * ((length + 1) // 2)
