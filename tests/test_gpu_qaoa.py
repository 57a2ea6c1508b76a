"""Batched QAOA entry point (include/orkan_batch.h) on the GPU.

Every instance of a batch is checked against the per-call plain path of the same library
(state_plus, exp_diag, rx on every qubit, mean -- the reference's own API, one call per
operation) and, where it finishes in seconds, against the oracle composition, at 1e-12.
"""
import numpy as np
import pytest

import orkan_b200
from oracle import restate as R
from orkan_b200.batch import QaoaBatch, erdos_renyi_graph, random_regular_graph

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def ork():
    return orkan_b200.load(5)


def graphs_for(ns, rng, weighted=False):
    edges, weights = [], []
    for n in ns:
        es = random_regular_graph(n, 3, rng) if n >= 4 else erdos_renyi_graph(n, 0.7, rng)
        edges.append(es)
        weights.append(rng.uniform(0.0, 1.0, len(es)) if weighted else np.ones(len(es)))
    return edges, (weights if weighted else None)


def angles(count, p, rng):
    return rng.uniform(0, np.pi, (count, p)), rng.uniform(0, np.pi / 2, (count, p))


def plain_mean(ork, n, cost, g, b):
    st = ork.plus("pure", n)
    for k in range(len(g)):
        ork.exp_diag(st, cost, float(g[k]))
        for q in range(n):
            ork.gate(st, "rx", [q], 2.0 * float(b[k]))
    m = ork.mean(st, cost)
    ork.free(st)
    return m


def costs_of(ns, edges, weights):
    return [R.maxcut_cost(n, e, None if weights is None else weights[i]) for i, (n, e) in enumerate(zip(ns, edges))]


@pytest.mark.parametrize("weighted", [False, True])
def test_uneven_small_batch_vs_oracle(ork, weighted):
    rng = np.random.default_rng(1 + weighted)
    ns = [1, 2, 3, 5, 7, 9, 11, 12, 13, 14, 15, 16, 4, 8, 6, 10]
    p = 3
    edges, weights = graphs_for(ns, rng, weighted)
    g, b = angles(len(ns), p, rng)
    with QaoaBatch(ork, ns, edges, weights, p) as bt:
        means = bt.run(g, b)
        for i, (n, cost) in enumerate(zip(ns, costs_of(ns, edges, weights))):
            assert abs(means[i] - R.qaoa_mean(n, cost, g[i], b[i])) < TOL, f"instance {i} (n={n})"


def test_cost_vectors_exact(ork):
    rng = np.random.default_rng(3)
    ns = [5, 12, 17]
    for weighted in (False, True):
        edges, weights = graphs_for(ns, rng, weighted)
        with QaoaBatch(ork, ns, edges, weights, 2) as bt:
            for i, cost in enumerate(costs_of(ns, edges, weights)):
                got = bt.cost_vector(i)
                if weighted:
                    assert np.abs(got - cost).max() < 1e-13
                else:
                    assert np.array_equal(got, cost)


def test_vs_plain_path(ork):
    rng = np.random.default_rng(5)
    ns = [16, 17, 18, 19, 20, 21, 16, 18]
    p = 4
    edges, _ = graphs_for(ns, rng)
    g, b = angles(len(ns), p, rng)
    with QaoaBatch(ork, ns, edges, None, p) as bt:
        means = bt.run(g, b)
        for i, (n, cost) in enumerate(zip(ns, costs_of(ns, edges, None))):
            assert abs(means[i] - plain_mean(ork, n, cost, g[i], b[i])) < TOL


def test_f64_costs_match_byte_costs(ork):
    rng = np.random.default_rng(7)
    ns = [14, 18, 9]
    edges, _ = graphs_for(ns, rng)
    g, b = angles(len(ns), 3, rng)
    with QaoaBatch(ork, ns, edges, None, 3) as b8, QaoaBatch(ork, ns, edges, None, 3, f64_costs=True) as b64:
        m8, m64 = b8.run(g, b), b64.run(g, b)
    assert np.abs(m8 - m64).max() < 1e-13


def test_waves_give_identical_results(ork):
    rng = np.random.default_rng(9)
    ns = [18, 17, 16, 16, 15, 14, 18, 17]
    p = 2
    edges, _ = graphs_for(ns, rng)
    g, b = angles(len(ns), p, rng)
    with QaoaBatch(ork, ns, edges, None, p) as one, \
            QaoaBatch(ork, ns, edges, None, p, mem_budget=(1 << 18) * 16) as many:
        assert one.stats()[0] == 1
        assert many.stats()[0] > 1
        assert np.array_equal(one.run(g, b), many.run(g, b))


def test_replays_are_deterministic(ork):
    rng = np.random.default_rng(11)
    ns = [20, 16, 12]
    edges, _ = graphs_for(ns, rng)
    g, b = angles(len(ns), 4, rng)
    with QaoaBatch(ork, ns, edges, None, 4) as bt:
        a = bt.run(g, b)
        g2, b2 = angles(len(ns), 4, rng)
        bt.run(g2, b2)
        assert np.array_equal(a, bt.run(g, b))


def test_shared_graph_many_angle_sets(ork):
    rng = np.random.default_rng(13)
    n, count, p = 15, 24, 3
    es = erdos_renyi_graph(n, 0.3, rng)
    w = rng.uniform(0, 1, len(es))
    cost = R.maxcut_cost(n, es, w)
    g, b = angles(count, p, rng)
    with QaoaBatch(ork, [n] * count, [es] * count, [w] * count, p) as bt:
        means = bt.run(g, b)
    for i in range(0, count, 5):
        assert abs(means[i] - R.qaoa_mean(n, cost, g[i], b[i])) < TOL


def test_tune_and_cache(ork, tmp_path):
    rng = np.random.default_rng(15)
    ns = [20, 19, 14, 18]
    p = 2
    edges, _ = graphs_for(ns, rng)
    g, b = angles(len(ns), p, rng)
    path = str(tmp_path / "tune.json")
    with QaoaBatch(ork, ns, edges, None, p) as bt:
        before = bt.run(g, b)
        bt.tune(g, b, path)
        for n in ns:
            C, t, ring = bt.config(n)
            assert t in (128, 256, 512) and ring in (1, 2) and C <= 13 and (C >= n or 2 * C >= n)
        after = bt.run(g, b)
        assert np.abs(after - before).max() < TOL
        lines = open(path).read().strip().splitlines()
        assert len(lines) == len(set(ns))
        chosen = {n: bt.config(n) for n in ns}
    with QaoaBatch(ork, ns, edges, None, p) as bt2:
        bt2.tune(g, b, path)                     # served from the cache: nothing appended
        assert open(path).read().strip().splitlines() == lines
        assert {n: bt2.config(n) for n in ns} == chosen
        assert np.abs(bt2.run(g, b) - before).max() < TOL


def test_regular_batch_every_instance_vs_plain_path(ork):
    """The 3-regular MaxCut batch shape (qubit counts uniform over 16..24, p = 4, gamma in
    [0, pi], beta in [0, pi/2]) at 48 instances; every instance against the plain path."""
    rng = np.random.default_rng(17)
    count, p = 48, 4
    ns = list(rng.integers(16, 25, count))
    edges, _ = graphs_for(ns, rng)
    g, b = angles(count, p, rng)
    with QaoaBatch(ork, ns, edges, None, p) as bt:
        means = bt.run(g, b)
        for i in range(count):
            cost = bt.cost_vector(i)
            assert abs(means[i] - plain_mean(ork, int(ns[i]), cost, g[i], b[i])) < TOL, f"instance {i}"


def test_sharded_batch_matches_the_whole_batch(ork):
    """The batch split over three ranks (here three shards on one GPU, no process group):
    each shard's means, scattered to their instance indices and summed, equal the whole
    batch's."""
    from orkan_b200.batch import ShardedQaoaBatch, scatter_means
    rng = np.random.default_rng(19)
    ns = [int(x) for x in rng.integers(10, 19, 30)]
    p = 3
    edges, _ = graphs_for(ns, rng)
    g, b = angles(len(ns), p, rng)
    with QaoaBatch(ork, ns, edges, None, p) as whole:
        want = whole.run(g, b)
    total = np.zeros(len(ns))
    seen = []
    for rank in range(3):
        sh = ShardedQaoaBatch(ork, ns, edges, None, p, rank=rank, world=3)
        loc = sh.run(g, b)
        assert len(loc) == len(sh.idx) > 0
        total += scatter_means(len(ns), sh.idx, loc)
        assert np.array_equal(sh.gather(loc), scatter_means(len(ns), sh.idx, loc))
        seen.extend(sh.idx.tolist())
        sh.close()
    assert sorted(seen) == list(range(len(ns)))
    assert np.abs(total - want).max() < TOL
