"""The sample-matrix oracle (oracle/sample.py) against the pinned per-call restatement:
its entries are <psi_a| diag(obs) |psi_b>, i.e. matel_diag (reference src/meas/meas_pure.c:32-46)
of independently built leaves, and mean on the diagonal."""
import numpy as np

from oracle import restate as R
from oracle import sample as SM


def _op(gates):
    def f(psi):
        for g, qs, th in gates:
            psi = R.apply_pure(psi, g, qs, th)
        return psi
    return f


def test_entries_are_matel_diag_of_the_leaves():
    rng = np.random.default_rng(1)
    n = 4
    iota = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    iota /= np.linalg.norm(iota)
    obs = rng.uniform(-1, 1, 1 << n)
    pre = ([_op([("h", [0], None)]), _op([("rx", [1], 0.3)])], [0.6, 0.8j])
    mid = ([_op([("x", [2], None)]), _op([("cz", [0, 3], None)]), _op([("ry", [3], 1.1), ("cx", [3, 1], None)])], None)
    post = ([_op([("t", [1], None)]), _op([("swap", [0, 2], None)])], [0.5 - 0.5j, 0.25])
    ch = [pre, mid, post]
    s = SM.sample_matrix(iota, obs, ch, 1)
    # leaves by hand
    p = 0.6 * R.apply_pure(iota.copy(), "h", [0]) + 0.8j * R.apply_pure(iota.copy(), "rx", [1], 0.3)
    leaves = []
    for op in mid[0]:
        v = op(p.copy())
        v = (0.5 - 0.5j) * R.apply_pure(v.copy(), "t", [1]) + 0.25 * R.apply_pure(v.copy(), "swap", [0, 2])
        leaves.append(v)
    for a in range(3):
        for b in range(3):
            assert abs(s[a, b] - R.matel_diag(leaves[a], leaves[b], obs)) < 1e-13
        assert abs(s[a, a].real - R.mean("pure", leaves[a], obs)) < 1e-13
    assert np.allclose(s, s.conj().T, atol=1e-14)
