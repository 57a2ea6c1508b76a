"""Parity at the benchmark configurations, against the reference library itself.

The reference (oracle/_ref/liborkan_ref_t5.so, compiled from the reference's own sources)
runs on the host cores beside the CUDA library on the same initial states, and the whole
storage arrays are compared at 1e-12 max-abs:

* 14-qubit tiled and packed density matrices (Dirichlet(1,1,1,1) mixtures of 4 Gaussian
  states, the single-gate sweep's states): every 4th sweep gate (at least 60) covering all
  18 gate calls, applied in sequence.  The two tiled patterns where the reference's tiled
  backend deviates from its own documented semantics (swap with both qubits >= LOG_TILE_DIM,
  ccx with all three) are compared against the reference's packed backend instead, at 10
  qubits, where full matrices are small;
* 13-qubit tiled and packed density matrices: the whole 52-channel set (depolarizing,
  amplitude and phase damping, random 4-Kraus CPTP channel on every qubit), then mean of a
  U[-1, 1] observable, and matel_diag on two 13-qubit statevectors;
* the 30-qubit statevector (16 GiB): 13 gates of the sweep, compared in 1 GiB pieces.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import restate as R
from orkan_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12
_LIBC = C.CDLL("libc.so.6")
_LIBC.malloc.restype = C.c_void_p
_LIBC.malloc.argtypes = [C.c_size_t]


def ref_from_device(ref, ork, st, kind, n):
    """A reference state holding a copy of a device state (no intermediate host copy: the
    storage is downloaded straight into a malloc'd buffer that the reference then owns)."""
    from oracle.ref import KIND, StateT
    nbytes = int(ork.lib.state_len(C.byref(st))) * 16
    buf = _LIBC.malloc(nbytes)
    assert buf, "host allocation failed"
    assert ork.lib.orkan_state_download(C.byref(st), C.c_void_p(buf)) == 0
    s = StateT(KIND[kind], None, 0)
    p = C.c_void_p(buf)
    ref.lib.state_init(C.byref(s), n, C.byref(p))
    return s


def max_diff(ork, st, ref, rs, chunk=1 << 26):
    """max |device storage - reference storage|, compared piece by piece."""
    count = int(ork.lib.state_len(C.byref(st)))
    view = W.state_view(ork, st)
    err = 0.0
    for off in range(0, count, chunk):
        m = min(chunk, count - off)
        dev = view[off:off + m].cpu().numpy()
        host = np.frombuffer((C.c_double * (2 * m)).from_address(rs.data + 16 * off), dtype=np.complex128)
        err = max(err, float(np.abs(dev - host).max()))
    return err


def tiled_defect(name, qs, lt=5):
    return (name == "swap" and min(qs) >= lt) or (name == "ccx" and min(qs) >= lt)


@pytest.mark.parametrize("kind", ["tiled", "packed"])
def test_sweep_subset_14q_against_reference(ork5, ref5, kind):
    n = 14
    plan = [g for g in W.sweep(n)[::4] if not (kind == "tiled" and tiled_defect(g[0], g[1]))]
    assert len(plan) >= 50 and len({g[0] for g in plan}) == 18
    st = ork5.state(kind, n)
    W.fill_state_on_device(ork5, st, kind, n, seed=1, log_tile=5)
    rs = ref_from_device(ref5, ork5, st, kind, n)
    for name, qs, th in plan:
        ork5.gate(st, name, qs, th)
        ref5.gate(rs, name, qs, th)
    err = max_diff(ork5, st, ref5, rs)
    ork5.free(st)
    ref5.free(rs)
    assert err <= TOL


def test_tiled_defect_patterns_against_reference_packed(ork5, ref5):
    """Where the reference's tiled swap/ccx deviate, the CUDA tiled result equals the
    reference's packed result (its documented semantics)."""
    n = 10
    rho = W.dirichlet_mixture(n, seed=21)
    gates = [("swap", (5, 9)), ("swap", (9, 6)), ("ccx", (5, 7, 9)), ("ccx", (9, 8, 5)), ("swap", (7, 8))]
    st = ork5.state("tiled", n, R.to_storage("tiled", rho, 5))
    rs = ref5.state("packed", n, R.to_storage("packed", rho, 5))
    for name, qs in gates:
        assert tiled_defect(name, qs)
        ork5.gate(st, name, qs)
        ref5.gate(rs, name, qs)
    want = R.to_storage("tiled", R.from_storage("packed", ref5.storage(rs), n, 5), 5)
    err = np.abs(ork5.storage(st) - want).max()
    ork5.free(st)
    ref5.free(rs)
    assert err <= TOL


def test_channel_set_13q_against_reference(ork5, ref5):
    import torch
    n = 13
    chans = W.channel_set(n, seed=3)
    assert len(chans) == 52
    obs = W.uniform_obs(n, seed=9)
    for kind in ("tiled", "packed"):
        st = ork5.state(kind, n)
        W.fill_state_on_device(ork5, st, kind, n, seed=5, log_tile=5)
        rs = ref_from_device(ref5, ork5, st, kind, n)
        for label, kraus, q in chans:
            ork5.channel_1q(st, ork5.superop(kraus), q)
            ref5.channel_1q(rs, ref5.superop(kraus), q)
        err = max_diff(ork5, st, ref5, rs)
        m_dev, m_ref = ork5.mean(st, obs), ref5.mean(rs, obs)
        ork5.free(st)
        ref5.free(rs)
        assert err <= TOL, kind
        assert abs(m_dev - m_ref) <= TOL, kind
    bra, ket = ork5.state("pure", n), ork5.state("pure", n)
    W.fill_state_on_device(ork5, bra, "pure", n, seed=6, log_tile=5)
    W.fill_state_on_device(ork5, ket, "pure", n, seed=7, log_tile=5)
    rb, rk = ref_from_device(ref5, ork5, bra, "pure", n), ref_from_device(ref5, ork5, ket, "pure", n)
    dev = ork5.matel_diag(bra, ket, obs)
    host = ref5.matel_diag(rb, rk, obs)
    for s in (bra, ket):
        ork5.free(s)
    for s in (rb, rk):
        ref5.free(s)
    torch.cuda.synchronize()
    assert abs(dev - host) <= TOL


def test_sweep_subset_30q_against_reference(ork5, ref5):
    n = 30
    plan = W.sweep(n)[::45]
    assert len(plan) >= 10
    st = ork5.state("pure", n)
    W.fill_state_on_device(ork5, st, "pure", n, seed=1, log_tile=5)
    rs = ref_from_device(ref5, ork5, st, "pure", n)
    for name, qs, th in plan:
        ork5.gate(st, name, qs, th)
        ref5.gate(rs, name, qs, th)
    err = max_diff(ork5, st, ref5, rs)
    ork5.free(st)
    ref5.free(rs)
    assert err <= TOL


@pytest.mark.parametrize("lt", [3, 5])
def test_matrix_gates_against_reference(request, lt):
    """single_from_mat / two_from_mat on tiled states: every target and every ordered pair
    at 7 qubits, CUDA library against the reference library directly."""
    ork, ref = request.getfixturevalue(f"ork{lt}"), request.getfixturevalue(f"ref{lt}")
    n = 7
    rng = np.random.default_rng(40 + lt)
    rho = W.dirichlet_mixture(n, seed=lt)
    st = ork.state("tiled", n, R.to_storage("tiled", rho, lt))
    rs = ref.state("tiled", n, R.to_storage("tiled", rho, lt))
    for q in range(n):
        u, _ = np.linalg.qr(rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2)))
        ork.single_from_mat(st, q, u.reshape(-1, order="F"))
        ref.single_from_mat(rs, q, u.reshape(-1, order="F"))
    for q1 in range(n):
        for q2 in range(n):
            if q1 == q2:
                continue
            u, _ = np.linalg.qr(rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)))
            ork.two_from_mat(st, q1, q2, u.reshape(-1, order="F"))
            ref.two_from_mat(rs, q1, q2, u.reshape(-1, order="F"))
    err = np.abs(ork.storage(st) - ref.storage(rs)).max()
    ork.free(st)
    ref.free(rs)
    assert err <= TOL
