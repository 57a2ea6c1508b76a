"""GPU parity: the CUDA library, called through its public C API (ctypes on
liborkan_b200.so / liborkan_b200_t3.so), against the oracle.

Tolerance: 1e-12 max-abs over the WHOLE storage array (diagonal-tile mirrors and tiled
padding included), the parity bar of the reference's own tests (test/include/test.h:40).
Sweeps follow the reference test strategy: every gate, every ordered qubit tuple, every
layout, both tile geometries (LOG_TILE_DIM 3 exercises multi-tile paths at 4-7 qubits).
"""
import itertools

import numpy as np
import pytest

from oracle import restate as R
from orkan_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rand_rho(n, seed, rank=3):
    rng = np.random.default_rng(seed)
    d = 1 << n
    a = rng.standard_normal((d, rank)) + 1j * rng.standard_normal((d, rank))
    rho = a @ a.conj().T
    return rho / np.trace(rho).real


def lib_for(request, lt):
    return request.getfixturevalue(f"ork{lt}")


def gate_cases(n, seed, max_3q=80):
    rng = np.random.default_rng(seed)
    for g in W.ALL_GATES:
        k = W.gate_arity(g)
        if k > n:
            continue
        tuples = list(itertools.permutations(range(n), k))
        if k == 3 and len(tuples) > max_3q:
            tuples = [tuples[i] for i in rng.choice(len(tuples), max_3q, replace=False)]
        for qs in tuples:
            theta = float(rng.uniform(0, 2 * np.pi)) if g in W.GATES_ROT else None
            yield g, qs, theta


@pytest.mark.parametrize("lt", [3, 5])
@pytest.mark.parametrize("kind", ["pure", "packed", "tiled"])
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7])
def test_every_gate_every_qubit_tuple(request, lt, kind, n):
    ork = lib_for(request, lt)
    full = W.gaussian_pure(n, 10 + n) if kind == "pure" else rand_rho(n, 10 + n)
    st = ork.state(kind, n, R.to_storage(kind, full, lt))
    start = R.to_storage(kind, full, lt)
    for g, qs, th in gate_cases(n, seed=n):
        ork.upload(st, start)
        ork.gate(st, g, qs, th)
        exp = R.to_storage(kind, R.apply_gate(kind, full, g, qs, th), lt)
        err = np.abs(ork.storage(st) - exp).max()
        assert err <= TOL, (g, qs, err)
    ork.free(st)


@pytest.mark.parametrize("lt", [3, 5])
@pytest.mark.parametrize("kind,n", [("pure", 12), ("packed", 8), ("tiled", 8)])
def test_random_circuit_config(request, lt, kind, n):
    """Parity configuration: 12 q PURE |+>, 8 q packed and tiled |+><+|, the same random
    200-gate circuit, then mean of a uniform [-1, 1] observable."""
    ork = lib_for(request, lt)
    circ = W.random_circuit(n, 200, seed=2024)
    obs = W.uniform_obs(n, seed=7)
    st = ork.plus(kind, n)
    full = R.plus_state(kind, n)
    assert np.abs(ork.storage(st) - R.to_storage(kind, full, lt)).max() <= TOL
    for g, qs, th in circ:
        ork.gate(st, g, qs, th)
        full = R.apply_gate(kind, full, g, qs, th)
    assert np.abs(ork.storage(st) - R.to_storage(kind, full, lt)).max() <= TOL
    assert abs(ork.mean(st, obs) - R.mean(kind, full, obs)) <= TOL
    ork.free(st)


@pytest.mark.parametrize("n", [14, 18, 20])
def test_pure_sweep_larger(ork5, n):
    psi = W.gaussian_pure(n, n)
    st = ork5.state("pure", n, psi)
    for g, qs, th in W.sweep(n)[:: 3]:
        ork5.gate(st, g, qs, th)
        psi = R.apply_pure(psi, g, qs, th)
    assert np.abs(ork5.storage(st) - psi).max() <= TOL
    ork5.free(st)


@pytest.mark.parametrize("lt", [3, 5])
@pytest.mark.parametrize("kind", ["packed", "tiled"])
def test_mixed_sweep_larger(request, lt, kind):
    ork = lib_for(request, lt)
    n = 10
    rho = W.dirichlet_mixture(n, seed=3)
    st = ork.state(kind, n, R.to_storage(kind, rho, lt))
    for g, qs, th in W.sweep(n)[:: 4]:
        ork.gate(st, g, qs, th)
        rho = R.apply_mixed(rho, g, qs, th)
    assert np.abs(ork.storage(st) - R.to_storage(kind, rho, lt)).max() <= TOL
    ork.free(st)


@pytest.mark.parametrize("lt", [3, 5])
@pytest.mark.parametrize("kind", ["packed", "tiled"])
def test_channels(request, lt, kind):
    ork = lib_for(request, lt)
    rng = np.random.default_rng(5)
    for n in (1, 2, 3, 6, 9):
        rho = rand_rho(n, 60 + n)
        st = ork.state(kind, n, R.to_storage(kind, rho, lt))
        a = rng.standard_normal((8, 2)) + 1j * rng.standard_normal((8, 2))
        iso, _ = np.linalg.qr(a)
        cptp = [iso[2 * i:2 * i + 2, :] for i in range(4)]
        for kr in (R.depolarizing_kraus(0.09), R.amplitude_damping_kraus(0.2), R.phase_damping_kraus(0.13), cptp):
            sop = ork.superop(kr)
            assert np.abs(sop - R.kraus_to_superop(kr)).max() <= TOL
            for q in range(n):
                ork.channel_1q(st, sop, q)
                rho = R.apply_superop1(rho, sop, q)
        assert np.abs(ork.storage(st) - R.to_storage(kind, rho, lt)).max() <= TOL
        ork.free(st)


@pytest.mark.parametrize("lt", [3, 5])
@pytest.mark.parametrize("kind", ["packed", "tiled"])
def test_channel_2q(request, lt, kind):
    """2-qubit channels (channel_2q, an extension: the reference's channel_1q is 1-local):
    kraus_to_superop of a random 4-term 2-qubit CPTP map, applied on ordered qubit pairs,
    against the oracle's restatement (itself checked against the Kraus sum)."""
    ork = lib_for(request, lt)
    rng = np.random.default_rng(8)
    for n in (2, 3, 5, 7):
        rho = rand_rho(n, 80 + n)
        st = ork.state(kind, n, R.to_storage(kind, rho, lt))
        iso, _ = np.linalg.qr(rng.standard_normal((16, 4)) + 1j * rng.standard_normal((16, 4)))
        kr = [iso[4 * i:4 * i + 4, :] for i in range(4)]
        sop = ork.superop(kr)
        assert np.abs(sop - R.kraus_to_superop(kr)).max() <= TOL
        pairs = list(itertools.permutations(range(n), 2))
        if len(pairs) > 20:
            pairs = [pairs[i] for i in rng.choice(len(pairs), 20, replace=False)]
        for q0, q1 in pairs:
            ork.channel_2q(st, sop, int(q0), int(q1))
            rho = R.apply_superop2(rho, sop, q0, q1)
        assert np.abs(ork.storage(st) - R.to_storage(kind, rho, lt)).max() <= TOL
        ork.free(st)


@pytest.mark.parametrize("lt", [3, 5])
@pytest.mark.parametrize("kind", ["packed", "tiled"])
def test_channel_2q_10q(request, lt, kind):
    """2-qubit channels at 10 qubits, where every engine geometry takes the FP64 tensor-core
    form (both qubits inside a sub-tile, one or both above it, adjacent and spread, either
    order), against the oracle's restatement."""
    ork = lib_for(request, lt)
    rng = np.random.default_rng(21)
    n = 10
    rho = rand_rho(n, 321)
    st = ork.state(kind, n, R.to_storage(kind, rho, lt))
    iso, _ = np.linalg.qr(rng.standard_normal((16, 4)) + 1j * rng.standard_normal((16, 4)))
    sop = ork.superop([iso[4 * i:4 * i + 4, :] for i in range(4)])
    for q0, q1 in ((0, 1), (1, 0), (0, 9), (9, 0), (2, 7), (5, 6), (8, 9), (9, 4), (3, 4)):
        ork.channel_2q(st, sop, q0, q1)
        rho = R.apply_superop2(rho, sop, q0, q1)
    assert np.abs(ork.storage(st) - R.to_storage(kind, rho, lt)).max() <= TOL
    ork.free(st)


@pytest.mark.parametrize("lt", [3, 5])
@pytest.mark.parametrize("kind", ["pure", "packed", "tiled"])
def test_mean_exp_diag(request, lt, kind):
    ork = lib_for(request, lt)
    for n in (1, 2, 5, 8, 11):
        rng = np.random.default_rng(n)
        full = W.gaussian_pure(n, n) if kind == "pure" else rand_rho(n, n)
        st = ork.state(kind, n, R.to_storage(kind, full, lt))
        obs = rng.uniform(-1, 1, size=1 << n)
        diag = rng.uniform(-5, 5, size=1 << n)
        m1 = ork.mean(st, obs)
        assert abs(m1 - R.mean(kind, full, obs)) <= TOL
        assert ork.mean(st, obs) == m1                                   # deterministic reduction
        ork.exp_diag(st, diag, 0.0)                                      # t == 0 is a no-op
        ork.exp_diag(st, diag, -1.21)
        full = R.exp_diag(kind, full, diag, -1.21)
        assert np.abs(ork.storage(st) - R.to_storage(kind, full, lt)).max() <= TOL
        ork.free(st)


def test_matel_diag(ork5):
    for n in (1, 4, 10, 16):
        rng = np.random.default_rng(n)
        bra, ket = W.gaussian_pure(n, n), W.gaussian_pure(n, n + 99)
        obs = rng.uniform(-1, 1, size=1 << n)
        sb, sk = ork5.state("pure", n, bra), ork5.state("pure", n, ket)
        assert abs(ork5.matel_diag(sb, sk, obs) - R.matel_diag(bra, ket, obs)) <= TOL
        ork5.free(sb)
        ork5.free(sk)


def test_known_answers(ork5):
    # <x> on |+>^n = (2^n - 1) / 2 ; matel -i/2 ; exp_diag on |k> ; single tile rho[1][0] = -0.5i
    for n in range(1, 5):
        s = ork5.plus("pure", n)
        assert abs(ork5.mean(s, np.arange(1 << n, dtype=float)) - ((1 << n) - 1) / 2) <= TOL
        ork5.free(s)
    bra = ork5.state("pure", 1, np.array([R.SQRT1_2, 1j * R.SQRT1_2]))
    ket = ork5.state("pure", 1, np.array([R.SQRT1_2, R.SQRT1_2]))
    assert abs(ork5.matel_diag(bra, ket, np.array([0.0, 1.0])) + 0.5j) <= TOL
    ork5.free(bra)
    ork5.free(ket)
    for k in range(4):
        s = ork5.state("pure", 2)
        ork5.set(s, k, 0, 1.0)
        ork5.exp_diag(s, np.arange(4, dtype=float), 1.0)
        assert abs(ork5.get(s, k) - (np.cos(k) - 1j * np.sin(k))) <= TOL
        ork5.free(s)
    s = ork5.plus("tiled", 1)
    ork5.exp_diag(s, np.array([0.0, 1.0]), np.pi / 2)
    assert abs(ork5.get(s, 1, 0) + 0.5j) <= TOL
    assert abs(ork5.get(s, 0, 1) - 0.5j) <= TOL
    ork5.free(s)


@pytest.mark.parametrize("lt", [3, 5])
def test_state_api(request, lt):
    ork = lib_for(request, lt)
    for kind, n in (("pure", 3), ("packed", 4), ("tiled", 2), ("tiled", 6)):
        full = W.gaussian_pure(n, 1) if kind == "pure" else rand_rho(n, 1)
        st = ork.state(kind, n, R.to_storage(kind, full, lt))
        cp = ork.copy(st)
        assert np.array_equal(ork.storage(cp), ork.storage(st))
        d = 1 << n
        for r in range(d):
            for c in ([0] if kind == "pure" else range(d)):
                assert abs(ork.get(st, r, c) - (full[r] if kind == "pure" else full[r, c])) <= TOL
        if kind != "pure":
            ork.set(cp, 0, d - 1, 0.25 + 0.5j)                 # upper-triangle write stores the conjugate
            assert abs(ork.get(cp, d - 1, 0) - (0.25 - 0.5j)) <= TOL
            full2 = full.copy()
            full2[0, d - 1], full2[d - 1, 0] = 0.25 + 0.5j, 0.25 - 0.5j
            assert np.abs(ork.storage(cp) - R.to_storage(kind, full2, lt)).max() <= TOL
        ork.free(cp)
        ork.free(st)
        ork.free(st)                                             # state_free is idempotent


def test_generic_unitaries(ork3):
    rng = np.random.default_rng(11)
    n = 6
    for kind in ("packed", "tiled"):
        rho = rand_rho(n, 8)
        st = ork3.state(kind, n, R.to_storage(kind, rho, 3))
        for q in range(n):
            u, _ = np.linalg.qr(rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2)))
            ork3.single_from_mat(st, q, np.asfortranarray(u).reshape(-1, order="F"))
            rho = R.conjugate_by(rho, u, [q], n)
        for q1, q2 in itertools.permutations(range(n), 2):
            u, _ = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))
            ork3.two_from_mat(st, q1, q2, u.reshape(-1, order="F"))
            rho = R.conjugate_by(rho, u, [max(q1, q2), min(q1, q2)], n)
        assert np.abs(ork3.storage(st) - R.to_storage(kind, rho, 3)).max() <= TOL
        ork3.free(st)


# ---- size-independent properties at the benchmark sizes -------------------------------
def test_full_size_pure_30q_properties(ork5):
    """30 q statevector (16 GiB): norm preserved by every gate, gates followed by their
    inverses restore the state's observables, mean is deterministic."""
    n = 30
    st = ork5.plus("pure", n)
    ones = np.ones(1 << n)
    obs = np.random.default_rng(3).uniform(-1, 1, size=1 << n)
    for g, qs, th in [("h", (0,), None), ("rx", (29,), 0.4), ("cx", (0, 29), None), ("ccx", (29, 14, 0), None),
                      ("t", (7,), None), ("ry", (15,), 1.3), ("swap", (3, 28), None), ("cy", (28, 1), None)]:
        ork5.gate(st, g, qs, th)
    assert abs(ork5.mean(st, ones) - 1.0) <= 1e-10
    m = ork5.mean(st, obs)
    assert ork5.mean(st, obs) == m
    for g, qs, th in reversed([("h", (0,), None), ("rx", (29,), 0.4), ("cx", (0, 29), None),
                               ("ccx", (29, 14, 0), None), ("tdg", (7,), None), ("ry", (15,), 1.3),
                               ("swap", (3, 28), None), ("cy", (28, 1), None)]):
        ork5.gate(st, g, qs, -th if th is not None else None)
    # back to |+>: mean of the uniform observable equals its average
    assert abs(ork5.mean(st, obs) - obs.mean()) <= 1e-10
    ork5.free(st)


@pytest.mark.parametrize("kind", ["packed", "tiled"])
def test_full_size_mixed_14q_properties(ork5, kind):
    """14 q density matrix (2.15 GB): trace preserved by gates and channels, a gate and its
    inverse restore the state (round trip against the uploaded storage)."""
    n = 14
    rng = np.random.default_rng(4)
    w, psis = W.dirichlet_mixture_terms(n, seed=5)
    # build the storage without the 4 GB full matrix
    if kind == "packed":
        r, c = R._packed_rc(n)
        live = np.ones(r.shape, dtype=bool)
    else:
        r, c, live = R._tiled_rc(n, 5)
    start = np.zeros(r.shape[0], dtype=np.complex128)
    for wi, p in zip(w, psis):
        start[live] += wi * p[r[live]] * np.conj(p[c[live]])
    st = ork5.state(kind, n, start)
    ones = np.ones(1 << n)
    seq = [("h", (13,), None), ("rx", (0,), 0.77), ("cx", (13, 2), None), ("swap", (12, 6), None),
           ("ccx", (13, 12, 11), None), ("cy", (5, 13), None), ("s", (9,), None)]
    for g, qs, th in seq:
        ork5.gate(st, g, qs, th)
    sop = ork5.superop(R.depolarizing_kraus(0.05))
    ork5.channel_1q(st, sop, 13)
    assert abs(ork5.mean(st, ones) - 1.0) <= 1e-10
    ork5.free(st)
    st = ork5.state(kind, n, start)
    for g, qs, th in seq:
        ork5.gate(st, g, qs, th)
    inv = {"s": "sdg"}
    for g, qs, th in reversed(seq):
        ork5.gate(st, inv.get(g, g), qs, -th if th is not None else None)
    assert np.abs(ork5.storage(st) - start).max() <= 1e-12
    ork5.free(st)


@pytest.mark.parametrize("kind", ["packed", "tiled"])
def test_engine_pipeline_many_items_per_block(ork5, kind):
    """12 q density matrices: thousands of engine work items, so every block runs its
    double-buffered pipeline over many items (small states give each block at most one)."""
    n = 12
    rng = np.random.default_rng(21)
    rho = rand_rho(n, 31)
    st = ork5.state(kind, n, R.to_storage(kind, rho, 5))
    seq = [("h", (0,), None), ("h", (11,), None), ("rx", (6,), 0.3), ("ry", (3,), 1.1), ("x", (9,), None),
           ("y", (1,), None), ("cx", (11, 0), None), ("cx", (2, 10), None), ("cy", (7, 8), None),
           ("swap", (11, 5), None), ("swap", (1, 2), None), ("ccx", (11, 10, 0), None), ("ccx", (0, 1, 9), None)]
    for g, qs, th in seq:
        ork5.gate(st, g, qs, th)
        rho = R.apply_mixed(rho, g, qs, th)
    sop = R.kraus_to_superop(R.amplitude_damping_kraus(0.3))
    for q in (0, 7, 11):
        ork5.channel_1q(st, sop, q)
        rho = R.apply_superop1(rho, sop, q)
    u, _ = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))
    ork5.two_from_mat(st, 11, 4, u.reshape(-1, order="F"))
    rho = R.conjugate_by(rho, u, [11, 4], n)
    assert np.abs(ork5.storage(st) - R.to_storage(kind, rho, 5)).max() <= TOL
    ork5.free(st)


def test_engine_reported_no_errors(ork5, ork3):
    """No density-matrix engine launch of this process ran out of its bounded wait for staged
    data (the kernel records that in an error word instead of waiting forever)."""
    for ork in (ork5, ork3):
        ork.lib.orkan_cu_engine_status.restype = __import__("ctypes").c_uint
        assert ork.lib.orkan_cu_engine_status() == 0

