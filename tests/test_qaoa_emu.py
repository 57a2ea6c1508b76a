"""Fused QAOA passes run by the CPU kernel emulator against the oracle composition.

The pass kernels (orkan_b200/csrc/cuda/qaoa.cuh) are executed thread by thread on the CPU
with a checking accessor: every access must stay in range, every amplitude must be written
exactly once per storing pass and read exactly once per loading pass, the state after each
pass must equal the oracle's circuit prefix, and the mean must match at 1e-12.
"""
import numpy as np
import pytest

import kemu
from oracle import restate as R


def graph(n, seed, weighted=False):
    rng = np.random.default_rng(seed)
    edges = [(u, v) for u in range(n) for v in range(u + 1, n) if rng.random() < 0.5]
    if not edges:
        edges = [(0, n - 1)] if n > 1 else []
    w = rng.uniform(0.1, 1.0, len(edges)) if weighted else None
    return edges, w


def angles(p, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(0, np.pi, p), rng.uniform(0, np.pi / 2, p)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8])
@pytest.mark.parametrize("p", [1, 2, 3])
@pytest.mark.parametrize("byte_cost", [True, False])
def test_full_pass_matches_oracle(n, p, byte_cost):
    edges, w = graph(n, 10 * n + p, weighted=not byte_cost)
    cost = R.maxcut_cost(n, edges, w)
    g, b = angles(p, n + 7 * p)
    res, m = kemu.qaoa(n, cost, p, g, b, log_chunk=max(n, 4), nthr=32, byte_cost=byte_cost)
    assert res.oob == 0
    assert res.reads.sum() == 0 and res.writes.sum() == 0      # a full pass keeps the state on chip
    assert abs(m - R.qaoa_mean(n, cost, g, b)) < 1e-12


CHUNKED = [(4, 2), (6, 3), (7, 4), (9, 5), (10, 5), (12, 7), (13, 8), (11, 11 // 2 + 1)]


@pytest.mark.parametrize("n,C", CHUNKED)
@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_passes_match_oracle_prefixes(n, C, p):
    byte_cost = (n + p) % 2 == 0
    edges, w = graph(n, 3 * n + p, weighted=not byte_cost)
    cost = R.maxcut_cost(n, edges, w)
    g, b = angles(p, 5 * n + p)
    for upto in range(p + 1):
        res, m = kemu.qaoa(n, cost, p, g, b, log_chunk=C, nthr=64, upto=upto, byte_cost=byte_cost)
        assert res.oob == 0
        stores = min(upto, p - 1) + 1
        loads = min(upto, p)
        assert np.all(res.writes == stores), "each storing pass writes every amplitude once"
        assert np.all(res.reads == loads), "each loading pass reads every amplitude once"
        if upto < p:
            half = "low" if upto % 2 == 0 else "high"
            want = R.qaoa_state(n, cost, g, b, low_qubits=C, layers=upto + 1, last_half=half)
            assert np.abs(res.out - want).max() < 1e-12
        else:
            assert abs(m - R.qaoa_mean(n, cost, g, b)) < 1e-12


@pytest.mark.parametrize("n,C,nthr", [(14, 13, 512), (13, 13, 512), (20, 12, 256), (17, 11, 128)])
def test_bench_chunk_shapes(n, C, nthr):
    """Chunk shapes of the GPU configurations: 2^13 chunks (a one-qubit group at slot bit
    12), 2^12 and 2^11 chunks with high passes of 8 and 6 row bits."""
    edges, _ = graph(n, 5)
    cost = R.maxcut_cost(n, edges)
    g, b = angles(2, 11)
    res, m = kemu.qaoa(n, cost, 2, g, b, log_chunk=C, nthr=nthr, byte_cost=True)
    assert res.oob == 0
    if n > C:
        assert np.all(res.writes == 2) and np.all(res.reads == 2)
    assert abs(m - R.qaoa_mean(n, cost, g, b)) < 1e-12


@pytest.mark.parametrize("nthr", [32, 96, 256])
def test_thread_counts(nthr):
    n, C, p = 10, 6, 3
    edges, _ = graph(n, 1)
    cost = R.maxcut_cost(n, edges)
    g, b = angles(p, 2)
    res, m = kemu.qaoa(n, cost, p, g, b, log_chunk=C, nthr=nthr, byte_cost=True)
    assert res.oob == 0
    assert abs(m - R.qaoa_mean(n, cost, g, b)) < 1e-12


def test_rejects_chunk_too_small():
    n = 9
    cost = R.maxcut_cost(n, [(0, 1)])
    with pytest.raises(RuntimeError):
        kemu.qaoa(n, cost, 1, [0.3], [0.2], log_chunk=4, nthr=32)


def test_regular_maxcut_is_integer_and_bounded():
    rng = np.random.default_rng(0)
    n = 12
    # a 3-regular graph by the configuration model with rejection
    while True:
        stubs = rng.permutation(np.repeat(np.arange(n), 3))
        pairs = stubs.reshape(-1, 2)
        if np.all(pairs[:, 0] != pairs[:, 1]) and len({tuple(sorted(p)) for p in pairs}) == len(pairs):
            break
    cost = R.maxcut_cost(n, [tuple(p) for p in pairs])
    assert np.all(cost == np.round(cost)) and cost.max() <= 3 * n // 2
    g, b = angles(4, 9)
    res, m = kemu.qaoa(n, cost, 4, g, b, log_chunk=7, nthr=64, byte_cost=True)
    assert res.oob == 0 and abs(m - R.qaoa_mean(n, cost, g, b)) < 1e-12


@pytest.mark.parametrize("n,C", [(6, 6), (11, 6)])
def test_mixer_forms_and_edge_angles(n, C):
    """beta = 0, pi/4 (|cos| = |sin|), pi/2 (cos = 0), and angles outside [0, pi/2] use both
    four-FMA forms of the rx update; gamma = 0 is the identity phase."""
    edges, _ = graph(n, 4)
    cost = R.maxcut_cost(n, edges)
    g = np.array([0.0, 0.7, np.pi, 2.5, -0.4])
    b = np.array([0.0, np.pi / 4, np.pi / 2, 3.0, -1.2])
    res, m = kemu.qaoa(n, cost, 5, g, b, log_chunk=C, nthr=32, byte_cost=True)
    assert res.oob == 0
    assert abs(m - R.qaoa_mean(n, cost, g, b)) < 1e-12


def test_shared_memory_regions_aligned_for_every_chunk():
    """Amplitude slots (16-byte asynchronous copies), cost words and the reduction array
    stay aligned for every chunk size and buffer depth (a misaligned region faults on the
    GPU, not on the CPU emulator)."""
    assert kemu.lib().emu_qaoa_smem_aligned() == 1
