"""Synthetic benchmark inputs (orkan_b200/workloads.py, orkan_b200/batch.py): the channel
configuration is trace preserving, the graphs have the promised degrees."""
import numpy as np
import pytest

from oracle import restate as R
from orkan_b200 import workloads as W
from orkan_b200.batch import erdos_renyi_graph, random_regular_graph


@pytest.mark.parametrize("n", [1, 5, 13])
def test_channel_set_is_cptp_on_every_qubit(n):
    chans = W.channel_set(n, seed=3)
    assert len(chans) == 4 * n and sorted({q for _, _, q in chans}) == list(range(n))
    for label, kr, q in chans:
        assert np.abs(sum(k.conj().T @ k for k in kr) - np.eye(2)).max() < 1e-14, label
        # its superoperator preserves the trace of any 2 x 2 block
        s = R.kraus_to_superop(kr)
        assert np.abs(s[0] + s[3] - np.array([1, 0, 0, 1])).max() < 1e-14


@pytest.mark.parametrize("n", list(range(4, 25)))
def test_regular_graphs(n):
    rng = np.random.default_rng(n)
    edges = random_regular_graph(n, 3, rng)
    deg = np.bincount(np.array(edges).ravel(), minlength=n)
    assert len({tuple(sorted(e)) for e in edges}) == len(edges) and all(u != v for u, v in edges)
    if n % 2 == 0:
        assert np.all(deg == 3)
    else:                                   # no 3-regular graph on an odd vertex count
        assert sorted(deg)[0] == 2 and np.all(np.array(sorted(deg)[1:]) == 3)


def test_erdos_renyi_graph():
    edges = erdos_renyi_graph(24, 0.3, np.random.default_rng(0))
    assert all(0 <= u < v < 24 for u, v in edges)
    assert 0.2 < len(edges) / (24 * 23 / 2) < 0.4
