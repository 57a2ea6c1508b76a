"""Host-side pieces of bench.py's JSON line (CPU only): the workload description both arms
share, the reference sample (the same fixed gates in the GPU arm's cpu_baseline and in every
step of the reference arm), the per-class DRAM traffic read from profiles/, and the
configured sizes of the learned legs."""
import os

import bench
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_both_arms_describe_the_same_workload():
    plan = bench.build_plan(12, 6)
    cfg = bench.sweep_config(12, 6, plan)
    assert cfg["gates_per_step"] == len(plan)
    assert cfg["algorithmic_bytes_per_step"] == sum(e[5] for e in plan)
    assert "12 q PURE" in cfg["workload"] and "6 q tiled and packed" in cfg["workload"]


def test_reference_sample_is_fixed_and_described():
    plan = bench.build_plan(30, 14)
    assert len(plan) == 1056
    txt = bench.sample_text(plan, 16, 7.5)
    assert f"every {bench.SAMPLE_STRIDE}th gate" in txt and "76 of 1056" in txt
    assert "30 q PURE, 14 q tiled, 14 q packed" in txt and "OpenMP threads = 16" in txt


def test_profiled_traffic_covers_the_sweep_classes():
    """The per-class DRAM traffic is read from the committed ncu summary's table."""
    prof = bench.profiled_traffic()
    classes = {bench.kernel_class(kind, name) for kind, _, name, *_ in bench.build_plan(8, 6)}
    assert classes <= set(prof)
    for c, (dram, alg) in prof.items():
        assert 0.8 < dram / alg < 2.0
    assert prof["pure_1q_dense"] == pytest.approx((4232.6e6, 4295.0e6))


def test_learned_legs_run_at_their_configured_sizes(monkeypatch):
    import sys
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse_args()
    assert a.surrogate_pairs == 65536 and a.noisy_pairs > 0
    assert a.batch_instances == 4096 and a.batch_check == -1 and a.circuit_gates == 200


def test_batched_cpu_baseline_times_every_qubit_count():
    """The batched leg's CPU baseline times the reference library on instances of every qubit
    count of the batch and weights each count's seconds per instance by its instances."""
    import numpy as np
    from oracle import ref
    if not ref.available(5):
        pytest.skip("the reference library (oracle/_ref) is not built")
    from orkan_b200.batch import random_regular_graph
    rng = np.random.default_rng(3)
    ns = np.array([4, 6, 4, 8, 6, 4, 8, 8])
    edges = [random_regular_graph(int(n), 3, rng) for n in ns]
    g = rng.uniform(0, np.pi, (len(ns), 2))
    b = rng.uniform(0, np.pi / 2, (len(ns), 2))
    out = bench.batched_cpu_baseline(ns, edges, g, b, 0.0)
    per = out["seconds_per_instance"]
    assert sorted(per) == ["4", "6", "8"]
    want = sum(int(np.sum(ns == n)) * per[str(n)] for n in (4, 6, 8))
    assert out["value"] == pytest.approx(len(ns) / want)
    assert "every qubit count" in out["sample"]
