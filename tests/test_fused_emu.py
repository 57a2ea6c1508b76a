"""The fused statevector kernel (k_pure_fused, orkan_b200/csrc/cuda/pure_fused.cuh) on the
CPU emulator: runs of gates cut the way the library's gate queue cuts them
(orkan_b200/csrc/host/fuse.c), including runs whose local qubits lie high, non-local
controls and non-local diagonal gates.  Every access stays in range, every amplitude is
loaded once and stored once per run, and the result equals the gates applied one by one --
bit for bit against the emulated one-gate kernels, and within 1e-12 of the oracle."""
import numpy as np
import pytest

import kemu
from oracle import restate as R
from orkan_b200 import workloads as W

TOL = 1e-12


def log_chunk_for(n):
    return n if n <= 12 else 11


def cut_runs(n, gates, cap=48, log_chunk=None):
    """The queue's greedy cut: a gate joins while the qubits it mixes plus qubits 0-2 fit
    the chunk and the run is below the cap."""
    lc = log_chunk or log_chunk_for(n)
    low = 7 if n >= 3 else (1 << n) - 1
    runs, cur, need = [], [], 0
    for g in gates:
        nd = kemu.fused_need(g[0], g[1]) | low
        if cur and (bin(need | nd).count("1") > lc or len(cur) >= cap):
            runs.append(cur)
            cur, need = [], 0
        if bin(nd).count("1") > lc:              # cannot be fused: launched on its own
            runs.append([g])
            continue
        cur.append(g)
        need |= nd
    if cur:
        runs.append(cur)
    return runs


def apply_one_by_one(psi, n, gates):
    for name, qs, th in gates:
        psi = kemu.pure_gate(psi, n, name, qs, th).out
    return psi


def check_runs(n, gates, log_chunk=None, grid_cap=0, cap=48):
    psi0 = W.gaussian_pure(n, 7 * n + len(gates))
    psi = psi0.copy()
    runs = cut_runs(n, gates, cap=cap, log_chunk=log_chunk)
    lc = log_chunk or log_chunk_for(n)
    low = 7 if n >= 3 else (1 << n) - 1
    for run in runs:
        if len(run) == 1 and bin(kemu.fused_need(run[0][0], run[0][1]) | low).count("1") > lc:
            psi = apply_one_by_one(psi, n, run)
            continue
        r = kemu.pure_fused(psi, n, lc, run, grid_cap)
        assert r.oob == 0
        assert (r.reads == 1).all() and (r.writes == 1).all()
        psi = r.out
    assert np.array_equal(psi, apply_one_by_one(psi0, n, gates))      # bit-identical
    want = psi0.copy()
    for name, qs, th in gates:
        want = R.apply_pure(want, name, qs, th)
    assert np.abs(psi - want).max() <= TOL
    return runs


@pytest.mark.parametrize("n", [1, 2, 3, 4, 6, 9])
def test_random_circuits_whole_state_chunk(n):
    gates = [g for g in W.random_circuit(max(n, 3), 300, seed=n) if max(g[1]) < n][:120]
    check_runs(n, gates)


@pytest.mark.parametrize("n,lc", [(8, 4), (9, 5), (10, 6), (11, 7), (13, 8)])
def test_random_circuits_small_chunks(n, lc):
    gates = W.random_circuit(n, 150, seed=100 + n)
    runs = check_runs(n, gates, log_chunk=lc, grid_cap=3)
    assert len(runs) < len(gates)


def test_high_local_qubits_and_nonlocal_controls():
    n, lc = 12, 7
    gates = [("h", (11,), None), ("rx", (9,), 0.7), ("cx", (1, 11), None), ("cx", (11, 4), None),
             ("cy", (10, 9), None), ("ccx", (10, 8, 11), None), ("ccx", (11, 9, 2), None),
             ("cz", (10, 8), None), ("cz", (11, 0), None), ("cz", (5, 3), None), ("rz", (10,), 1.3),
             ("rz", (9,), 0.4), ("p", (8,), 2.1), ("t", (6,), None), ("sdg", (11,), None),
             ("swap", (11, 0), None), ("swap", (9, 1), None), ("y", (2,), None), ("hy", (9,), None),
             ("s", (5,), None), ("tdg", (10,), None), ("z", (7,), None), ("ry", (11,), 2.9)]
    runs = check_runs(n, gates, log_chunk=lc, grid_cap=5)
    assert len(runs) == 1


@pytest.mark.parametrize("name", list(W.ALL_GATES))
def test_every_gate_on_every_tuple(name):
    n, lc = 5, 4
    k = W.gate_arity(name)
    rng = np.random.default_rng(3)
    import itertools
    for qs in itertools.permutations(range(n), k):
        th = float(rng.uniform(0, 2 * np.pi)) if name in W.GATES_ROT else None
        gates = [("h", (0,), None), (name, qs, th), ("t", (1,), None)]
        if bin(kemu.fused_need(name, qs) | 7).count("1") > lc:
            continue
        check_runs(n, gates, log_chunk=lc, grid_cap=2)


def test_queue_cut_respects_the_gate_cap():
    n = 10
    gates = W.random_circuit(n, 100, seed=5)
    runs = check_runs(n, gates, cap=7)
    assert max(len(r) for r in runs) <= 7


def test_register_stages_group_the_mixed_qubits():
    """A stage holds consecutive gates whose mixed local qubits fit a group of three: mixing
    gates on three distinct qubits and any number of diagonal gates and controls share one
    stage, a fourth distinct mixed qubit opens the next, and runs of random gates need far
    fewer stages than gates (each stage is one shared-memory round trip of the chunk)."""
    n = 12
    run = [("h", (1,), None), ("t", (9,), None), ("rx", (4,), 0.3), ("cz", (2, 7), None), ("y", (6,), None),
           ("rz", (11,), 0.2), ("cx", (3, 6), None), ("ccx", (9, 10, 4), None), ("p", (0,), 1.1)]
    assert kemu.fused_stages(n, 12, run) == 1
    assert kemu.fused_stages(n, 12, run + [("h", (10,), None)]) == 2
    gates = W.random_circuit(n, 48, seed=8)
    assert kemu.fused_stages(n, 12, gates) <= 48 // 3
