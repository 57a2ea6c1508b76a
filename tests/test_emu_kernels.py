"""CPU emulation of the CUDA kernels' index logic against the oracle (no GPU needed).

The same __host__ __device__ kernel functions that run on the B200 are executed on the
CPU by tests/emu/libkemu.so with a checking memory accessor.  For every gate, qubit tuple
and layout at small sizes this proves:
  * no access leaves the storage array (oob == 0);
  * the density-matrix engine reads every stored lower-triangle element exactly once,
    writes it exactly once, writes the tiled diagonal-tile mirrors exactly once and never
    reads them, and never touches the tiled padding;
  * the results equal the oracle (U rho U^dagger on the full matrix) to 1e-12.
"""
import itertools

import numpy as np
import pytest

import kemu
from oracle import restate as R
from orkan_b200 import traffic as T
from orkan_b200 import workloads as W

TOL = 1e-12
LAYOUTS = [("packed", 5), ("tiled", 3), ("tiled", 5)]


def rand_rho(n, seed):
    rng = np.random.default_rng(seed)
    d = 1 << n
    a = rng.standard_normal((d, 3)) + 1j * rng.standard_normal((d, 3))
    rho = a @ a.conj().T
    return rho / np.trace(rho).real


def storage_rc(kind, n, lt):
    if kind == "packed":
        r, c = R._packed_rc(n)
        return r, c, np.ones(r.shape, dtype=bool)
    return R._tiled_rc(n, lt)


def check_engine_counts(kind, n, lt, res, gate=None, qubits=None):
    """Every stored lower-triangle element the gate may change is read once and written
    once; the tiled diagonal-tile mirrors are never read and are written once when they
    may change; elements a monomial gate leaves in place are read and written at most once
    (whole lines of them are skipped; the oracle comparison checks their values); the tiled
    padding is never touched."""
    r, c, live = storage_rc(kind, n, lt)
    assert res.oob == 0
    changed = np.ones(r.shape, dtype=bool)
    if gate in ("cx", "cy", "swap", "ccx"):
        changed = T.mixed_changes(gate, qubits)(r, c)
    lower = live & (r >= c)
    upper = live & (r < c)
    assert np.all(res.reads[lower & changed] == 1)
    assert np.all(res.writes[lower & changed] == 1)
    assert np.all(res.reads[upper] == 0)
    assert np.all(res.writes[upper & changed] == 1)
    assert res.reads.max(initial=0) <= 1 and res.writes.max(initial=0) <= 1
    assert np.all(res.reads[~live] == 0) and np.all(res.writes[~live] == 0)


def check_phase_counts(kind, n, lt, res):
    r, c, live = storage_rc(kind, n, lt)
    assert res.oob == 0
    assert res.reads.max(initial=0) <= 1 and res.writes.max(initial=0) <= 1
    assert np.all(res.reads[r <= c] == 0)                       # diagonal and mirrors never read
    assert np.all(res.writes[(r == c) | ~live] == 0)            # diagonal and padding never written


def gate_cases(n, max_ccx=60, seed=0):
    rng = np.random.default_rng(seed)
    for g in W.ALL_GATES:
        k = W.gate_arity(g)
        if k > n:
            continue
        tuples = list(itertools.permutations(range(n), k))
        if k == 3 and len(tuples) > max_ccx:
            tuples = [tuples[i] for i in rng.choice(len(tuples), max_ccx, replace=False)]
        for qs in tuples:
            theta = float(rng.uniform(0, 2 * np.pi)) if g in W.GATES_ROT else None
            yield g, qs, theta


@pytest.mark.parametrize("kind,lt", LAYOUTS)
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 8])
def test_dm_gates_emulated(kind, lt, n):
    rho = rand_rho(n, 100 + n)
    st = R.to_storage(kind, rho, lt)
    for g, qs, theta in gate_cases(n, seed=n):
        res = kemu.dm_gate(kind, lt, st, n, g, qs, theta)
        exp = R.to_storage(kind, R.apply_mixed(rho, g, qs, theta), lt)
        err = np.abs(res.out - exp).max()
        assert err <= TOL, (g, qs, err)
        if g in ("z", "s", "sdg", "t", "tdg", "p", "rz", "cz"):
            check_phase_counts(kind, n, lt, res)
        else:
            check_engine_counts(kind, n, lt, res, g, qs)


@pytest.mark.parametrize("kind,lt", LAYOUTS)
@pytest.mark.parametrize("max_v", [8, 16])
def test_dm_monomials_small_blocks_emulated(kind, lt, max_v, monkeypatch):
    """Smaller block caps put more of a controlled flip's controls above the staged block
    (item-level conditions, unchanged items skipped) and more gate qubits on pairing bits."""
    monkeypatch.setenv("ORKAN_DM_MAX_V", str(max_v))
    n = 7
    rho = rand_rho(n, 300 + max_v)
    st = R.to_storage(kind, rho, lt)
    for g, qs, theta in gate_cases(n, max_ccx=120, seed=max_v):
        if g not in ("x", "y", "cx", "cy", "ccx", "swap"):
            continue
        res = kemu.dm_gate(kind, lt, st, n, g, qs, theta)
        exp = R.to_storage(kind, R.apply_mixed(rho, g, qs, theta), lt)
        assert np.abs(res.out - exp).max() <= TOL, (g, qs)
        check_engine_counts(kind, n, lt, res, g, qs)


@pytest.mark.parametrize("kind,lt", LAYOUTS)
@pytest.mark.parametrize("n", [2, 5, 7])
def test_dm_generic_unitaries_emulated(kind, lt, n):
    rng = np.random.default_rng(7 + n)
    rho = rand_rho(n, 200 + n)
    st = R.to_storage(kind, rho, lt)
    for k in (1, 2):
        for qs in itertools.permutations(range(n), k):
            a = rng.standard_normal((1 << k, 1 << k)) + 1j * rng.standard_normal((1 << k, 1 << k))
            u, _ = np.linalg.qr(a)
            res = kemu.dm_unitary(kind, lt, st, n, list(qs), u)
            exp = R.to_storage(kind, R.conjugate_by(rho, u, list(qs), n), lt)
            assert np.abs(res.out - exp).max() <= TOL
            check_engine_counts(kind, n, lt, res)


@pytest.mark.parametrize("kind,lt", LAYOUTS)
@pytest.mark.parametrize("n", [1, 3, 6, 7])
def test_dm_superop_emulated(kind, lt, n):
    rho = rand_rho(n, 300 + n)
    st = R.to_storage(kind, rho, lt)
    for kr in (R.depolarizing_kraus(0.07), R.amplitude_damping_kraus(0.15), R.phase_damping_kraus(0.1)):
        sop = R.kraus_to_superop(kr)
        for q in range(n):
            res = kemu.dm_superop1(kind, lt, st, n, q, sop)
            exp = R.to_storage(kind, R.apply_superop1(rho, sop, q), lt)
            assert np.abs(res.out - exp).max() <= TOL
            check_engine_counts(kind, n, lt, res)


def random_cptp_2q(rng, terms=4):
    """Kraus operators of a random 2-qubit channel: blocks of a 4*terms x 4 isometry."""
    a = rng.normal(size=(4 * terms, 4)) + 1j * rng.normal(size=(4 * terms, 4))
    q, _ = np.linalg.qr(a)
    return [q[4 * k:4 * k + 4, :] for k in range(terms)]


def test_superop2_oracle_is_the_kraus_sum():
    """The 2-qubit superoperator restatement against sum_a K_a rho K_a^dagger with the
    pinned Kronecker embedding (local index 2 bit(q0) + bit(q1), q0 the high bit)."""
    rng = np.random.default_rng(5)
    n = 4
    rho = rand_rho(n, 9)
    kr = random_cptp_2q(rng)
    sop = R.kraus_to_superop(kr)
    for q0, q1 in itertools.permutations(range(n), 2):
        want = sum(R.apply_left(R.apply_left(rho, k, [q0, q1], n).conj().T, k, [q0, q1], n).conj().T for k in kr)
        assert np.abs(R.apply_superop2(rho, sop, q0, q1) - want).max() < 1e-13


@pytest.mark.parametrize("max_v", ["8", "16", "32", "64"])
def test_superop2_fragment_staging_stays_in_the_block(max_v, monkeypatch):
    """Before its first item an engine block running channel_2q in the tensor-core form stages
    the 256 superoperator entries in its staged block: for every geometry of 2..14 qubits,
    both layouts and tile sizes and every block-side cap, the items that take that form have
    a staged block of at least 256 slots inside the block's dynamic shared memory."""
    import ctypes as C
    monkeypatch.setenv("ORKAN_DM_MAX_V", max_v)
    f = kemu.lib().emu_super2_geometry
    f.argtypes = [C.c_int, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.POINTER(C.c_uint64)]
    out = (C.c_uint64 * 3)()
    seen = set()
    for kind, lt in LAYOUTS:
        for n in range(2, 15):
            for q0, q1 in itertools.permutations(range(n), 2):
                r = f(kemu.LAYOUT[kind], lt, n, q0, q1, out)
                assert r >= 0, (kind, lt, n, q0, q1)
                V, P, smem = out[0], out[1], out[2]
                seen.add((r & 1, V))
                if r & 1:
                    assert r & 2 and V >= 16 and V * P >= 256, (kind, lt, n, q0, q1, V, P)
                    assert smem >= 16 + V * P * 16
    assert any(m for m, _ in seen) and any(not m for m, _ in seen)


@pytest.mark.parametrize("kind,lt", LAYOUTS)
@pytest.mark.parametrize("n", [2, 3, 5, 7])
def test_dm_superop2_emulated(kind, lt, n):
    rng = np.random.default_rng(40 + n)
    rho = rand_rho(n, 400 + n)
    st = R.to_storage(kind, rho, lt)
    sop = R.kraus_to_superop(random_cptp_2q(rng))
    pairs = list(itertools.permutations(range(n), 2))
    if len(pairs) > 24:
        pairs = [pairs[i] for i in rng.choice(len(pairs), 24, replace=False)]
    for q0, q1 in pairs:
        res = kemu.dm_superop2(kind, lt, st, n, q0, q1, sop)
        exp = R.to_storage(kind, R.apply_superop2(rho, sop, q0, q1), lt)
        assert np.abs(res.out - exp).max() <= TOL, (q0, q1)
        check_engine_counts(kind, n, lt, res)


@pytest.mark.parametrize("kind,lt", LAYOUTS)
@pytest.mark.parametrize("n", [1, 2, 4, 7])
def test_dm_exp_diag_emulated(kind, lt, n):
    rho = rand_rho(n, 400 + n)
    diag = np.random.default_rng(n).uniform(-3, 3, size=1 << n)
    st = R.to_storage(kind, rho, lt)
    res = kemu.dm_exp_diag(kind, lt, st, n, diag, 0.37)
    exp = R.to_storage(kind, R.exp_diag(kind, rho, diag, 0.37), lt)
    assert np.abs(res.out - exp).max() <= TOL
    check_phase_counts(kind, n, lt, res)


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 11])
def test_pure_gates_emulated(n):
    psi = W.gaussian_pure(n, 500 + n)
    for g, qs, theta in gate_cases(n, seed=n):
        res = kemu.pure_gate(psi, n, g, qs, theta)
        exp = R.apply_pure(psi, g, qs, theta)
        assert res.oob == 0
        assert res.reads.max() <= 1 and res.writes.max() <= 1
        assert np.abs(res.out - exp).max() <= TOL, (g, qs)
        if g in ("x", "y", "h", "hy", "rx", "ry", "rz"):
            assert np.all(res.reads == 1) and np.all(res.writes == 1)


@pytest.mark.parametrize("n", [1, 4, 10])
def test_pure_exp_diag_emulated(n):
    psi = W.gaussian_pure(n, 600 + n)
    diag = np.random.default_rng(n).uniform(-5, 5, size=1 << n)
    res = kemu.pure_exp_diag(psi, n, diag, 1.3)
    assert res.oob == 0 and np.all(res.reads == 1) and np.all(res.writes == 1)
    assert np.abs(res.out - R.exp_diag("pure", psi, diag, 1.3)).max() <= TOL


@pytest.mark.parametrize("kind,lt,n", [("pure", 5, 6), ("packed", 5, 5), ("tiled", 5, 3), ("tiled", 5, 7),
                                       ("tiled", 3, 2), ("tiled", 3, 6)])
def test_fill_emulated(kind, lt, n):
    d = 1 << n
    length = R.state_len(kind, n, lt)
    corner = (lt, d) if kind == "tiled" and d < (1 << lt) else (0, 0)
    res = kemu.fill(length, 0.25, *corner)
    assert res.oob == 0
    exp = R.to_storage(kind, np.full(d if kind == "pure" else (d, d), 0.25, dtype=complex), lt)
    assert np.array_equal(res.out, exp)


@pytest.mark.parametrize("lt", [6, 7])
@pytest.mark.parametrize("n", [3, 6, 8])
def test_tiles_larger_than_phase_subtile_emulated(lt, n):
    """Tile sides of 64 and 128 (LOG_TILE_DIM 6, 7): sub-tiles smaller than a tile, so
    off-diagonal sub-tiles of a diagonal tile need their mirror rewritten."""
    rng = np.random.default_rng(lt * 10 + n)
    rho = rand_rho(n, 700 + n)
    st = R.to_storage("tiled", rho, lt)
    for g in ("z", "t", "rz", "cz", "h", "cx", "swap", "ccx", "ry"):
        k = W.gate_arity(g)
        if k > n:
            continue
        qs = tuple(int(q) for q in rng.choice(n, k, replace=False))
        th = 0.4 if g in W.GATES_ROT else None
        res = kemu.dm_gate("tiled", lt, st, n, g, qs, th)
        exp = R.to_storage("tiled", R.apply_mixed(rho, g, qs, th), lt)
        assert res.oob == 0 and np.abs(res.out - exp).max() <= TOL, (g, qs)
    diag = rng.uniform(-2, 2, 1 << n)
    res = kemu.dm_exp_diag("tiled", lt, st, n, diag, 0.3)
    assert np.abs(res.out - R.to_storage("tiled", R.exp_diag("tiled", rho, diag, 0.3), lt)).max() <= TOL
