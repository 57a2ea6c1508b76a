"""sample_matrix (include/orkan_sample.h) on the GPU against the brute-force oracle
(oracle/sample.py): every leaf built independently on the CPU, S[a, b] a plain reduction.
Also the properties the specification asks for (reference docs/SAMPLE_MATRIX.md section 7):
Hermitian, real diagonal, the same result bit for bit whatever the workspace budget, the
prefix left in the input state, and the budget check."""
import os
import subprocess
import sys

import numpy as np
import pytest

import orkan_b200
from oracle import restate as R
from oracle import sample as SM
from orkan_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL = 1e-12
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def ork():
    return orkan_b200.load(5)


def random_gates(n, rng, count):
    out = []
    for _ in range(count):
        g = W.ALL_GATES[rng.integers(len(W.ALL_GATES))]
        k = W.gate_arity(g)
        if k > n:
            continue
        qs = [int(q) for q in rng.permutation(n)[:k]]
        th = float(rng.uniform(0, 2 * np.pi)) if g in W.GATES_ROT else None
        out.append((g, qs, th))
    return out


def make_op(ork, gates):
    def gpu(st):
        for g, qs, th in gates:
            ork.gate(st, g, qs, th)

    def cpu(psi):
        for g, qs, th in gates:
            psi = R.apply_pure(psi, g, qs, th)
        return psi
    return gpu, cpu


def ansatz(ork, n, sizes, at, rng):
    """Channels of the given sizes; weights random complex (None at `at`)."""
    gpu_ch, cpu_ch = [], []
    for l, k in enumerate(sizes):
        ops = [make_op(ork, random_gates(n, rng, int(rng.integers(1, 4)))) for _ in range(k)]
        w = None if l == at else (rng.normal(size=k) + 1j * rng.normal(size=k)) / np.sqrt(2 * k)
        gpu_ch.append(([o[0] for o in ops], w))
        cpu_ch.append(([o[1] for o in ops], w))
    return gpu_ch, cpu_ch


def setup(ork, n, seed):
    rng = np.random.default_rng(seed)
    iota = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    iota /= np.linalg.norm(iota)
    obs = rng.uniform(-1, 1, 1 << n)
    return rng, iota, obs


def run(ork, n, iota, obs, gpu_ch, at, budget):
    st = ork.state("pure", n, iota.astype(np.complex128))
    s = ork.sample_matrix(st, obs, gpu_ch, at, budget)
    pre = ork.storage(st)
    ork.free(st)
    return s, pre


@pytest.mark.parametrize("n,sizes,at", [(3, [2, 5, 3], 1), (4, [8], 0), (4, [3, 4, 2, 6], 3), (4, [5, 7, 2], 0)])
def test_brute_force_small(ork, n, sizes, at):
    rng, iota, obs = setup(ork, n, 10 * n + at + len(sizes))
    gpu_ch, cpu_ch = ansatz(ork, n, sizes, at, rng)
    s, _ = run(ork, n, iota, obs, gpu_ch, at, 1 << 30)
    want = SM.sample_matrix(iota, obs, cpu_ch, at)
    assert np.abs(s - want).max() < TOL


def test_larger_state_two_channels_after(ork):
    n = 12
    rng, iota, obs = setup(ork, n, 7)
    gpu_ch, cpu_ch = ansatz(ork, n, [3, 20, 4, 2], 1, rng)
    s, pre = run(ork, n, iota, obs, gpu_ch, 1, 1 << 30)
    assert np.abs(s - SM.sample_matrix(iota, obs, cpu_ch, 1)).max() < TOL
    # the input state holds the prefix K_0 |iota> on return
    want_pre = SM.apply_channel(cpu_ch[0][0], cpu_ch[0][1], iota.astype(np.complex128))
    assert np.abs(pre - want_pre).max() < TOL


def test_hermitian_real_diagonal_and_budget_independent(ork):
    n, K = 10, 37                       # several 16-column blocks
    rng, iota, obs = setup(ork, n, 3)
    gpu_ch, cpu_ch = ansatz(ork, n, [2, K, 3], 1, rng)
    vec = (1 << n) * 16
    results = [run(ork, n, iota, obs, gpu_ch, 1, b)[0] for b in (1 << 30, 4 * vec, 12 * vec, 30 * vec)]
    s = results[0]
    assert np.array_equal(s, s.conj().T)
    assert np.all(np.diag(s).imag == 0.0)
    for other in results[1:]:
        assert np.array_equal(other, s)
    assert np.abs(s - SM.sample_matrix(iota, obs, cpu_ch, 1)).max() < TOL


def test_workspace_below_four_vectors_is_rejected():
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import numpy as np, orkan_b200\n"
        "ork = orkan_b200.load(5)\n"
        "st = ork.plus('pure', 6)\n"
        "ork.sample_matrix(st, np.ones(64), [([lambda s: None, lambda s: None], None)], 0, 3 * 64 * 16)\n"
    ) % ROOT
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 1
    assert "orkan: sample_matrix: workspace too small" in r.stderr
