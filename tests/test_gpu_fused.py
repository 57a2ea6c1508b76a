"""Statevector gate fusion on the GPU (orkan_b200/csrc/host/fuse.c and k_pure_fused).

Gate calls on a PURE state are queued and applied in runs, one pass over device memory per
run.  These tests check, through the public C API:
* the 200-gate random circuit at 12 and 20 qubits against the oracle at 1e-12, and
  bit-identical to the same circuit with fusion off (every gate its own launch);
* a 30-qubit random circuit, fused against unfused, bit for bit (compared on the device);
* that every API call that reads the state sees the queued gates (mean, matel_diag,
  state_get, state_cp, exp_diag, download), that freeing a state drops its queue, and that
  fewer kernels launch with fusion on."""
import numpy as np
import pytest

from oracle import restate as R
from orkan_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12


def run_circuit(ork, n, gates, fusion):
    ork.set_gate_fusion(fusion)
    try:
        st = ork.plus("pure", n)
        l0 = ork.launches()
        for g, qs, th in gates:
            ork.gate(st, g, qs, th)
        ork.flush()
        launched = ork.launches() - l0
        out = ork.storage(st)
        ork.free(st)
    finally:
        ork.set_gate_fusion(48)
    return out, launched


@pytest.mark.parametrize("n", [12, 20])
def test_random_circuit_against_oracle_and_unfused(ork5, n):
    gates = W.random_circuit(n, 200, seed=1)
    fused, l_f = run_circuit(ork5, n, gates, 48)
    plain, l_p = run_circuit(ork5, n, gates, 0)
    assert np.array_equal(fused, plain)
    want = R.plus_state("pure", n)
    for g, qs, th in gates:
        want = R.apply_pure(want, g, qs, th)
    assert np.abs(fused - want).max() <= TOL
    assert l_p == 200
    assert l_f < l_p // 3


def test_random_circuit_30q_fused_equals_unfused(ork5):
    import torch
    n = 30
    gates = W.random_circuit(n, 60, seed=30)
    views = []
    states = []
    for fusion in (48, 0):
        ork5.set_gate_fusion(fusion)
        st = ork5.state("pure", n)
        W.fill_state_on_device(ork5, st, "pure", n, seed=3, log_tile=5)
        for g, qs, th in gates:
            ork5.gate(st, g, qs, th)
        states.append(st)
        views.append(W.state_view(ork5, st))
    ork5.set_gate_fusion(48)
    torch.cuda.synchronize()
    assert bool(torch.equal(views[0], views[1]))
    del views
    for st in states:
        ork5.free(st)


def test_every_reading_call_sees_queued_gates(ork5):
    n = 9
    gates = W.random_circuit(n, 40, seed=9)
    want = R.plus_state("pure", n)
    for g, qs, th in gates:
        want = R.apply_pure(want, g, qs, th)
    obs = W.uniform_obs(n, seed=2)
    ork5.set_gate_fusion(48)

    def fresh():
        st = ork5.plus("pure", n)
        for g, qs, th in gates:
            ork5.gate(st, g, qs, th)
        return st

    st = fresh()
    assert abs(ork5.mean(st, obs) - R.mean("pure", want, obs)) <= TOL
    ork5.free(st)
    st = fresh()
    assert abs(ork5.get(st, 5) - want[5]) <= TOL
    ork5.free(st)
    st = fresh()
    cp = ork5.copy(st)
    assert np.abs(ork5.storage(cp) - want).max() <= TOL
    ket = fresh()
    assert abs(ork5.matel_diag(st, ket, obs) - R.matel_diag(want, want, obs)) <= TOL
    for s in (st, cp, ket):
        ork5.free(s)
    st = fresh()
    ork5.exp_diag(st, obs, 0.6)
    assert np.abs(ork5.storage(st) - R.exp_diag("pure", want, obs, 0.6)).max() <= TOL
    ork5.free(st)
    # freeing a state with queued gates drops them; the next state is unaffected
    st = fresh()
    ork5.free(st)
    other = ork5.plus("pure", n)
    assert np.abs(ork5.storage(other) - R.plus_state("pure", n)).max() <= TOL
    ork5.free(other)
    # gates on two states interleaved
    a, b = ork5.plus("pure", n), ork5.plus("pure", n)
    wa, wb = R.plus_state("pure", n), R.plus_state("pure", n)
    for i, (g, qs, th) in enumerate(gates):
        s, = (a,) if i % 3 else (b,)
        ork5.gate(s, g, qs, th)
        if i % 3:
            wa = R.apply_pure(wa, g, qs, th)
        else:
            wb = R.apply_pure(wb, g, qs, th)
    assert np.abs(ork5.storage(a) - wa).max() <= TOL
    assert np.abs(ork5.storage(b) - wb).max() <= TOL
    ork5.free(a)
    ork5.free(b)
