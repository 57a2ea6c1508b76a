"""CPU restatement of Orkan's state-update path -- TEST INFRASTRUCTURE ONLY.

This module is the parity checker for the CUDA library.  Only tests/, the smoke check
in __graft_entry__.py and the cpu_baseline leg of bench.py may import it; the product
library never calls it.

What it restates (all in numpy, float64 / complex128):
  * storage layouts: packed lower-triangular column-major (reference src/internal/index.h:57-68,
    src/state/state_packed.c:1-54) and tiled (index.h:79-88, src/state/state_tiled.c:1-81), with
    both triangles stored in diagonal tiles and zero padding when 2^n < TILE_DIM;
  * gate matrices of the reference's tests (test/utility/gatemat.c:109-316,
    test/include/test_gate.h:100-210): local index with the first listed qubit as the most
    significant bit (gatemat.c:178-181);
  * PURE gates with the reference's pair formulas (src/gate/gate_pure.c:33-434);
  * mixed-state gates as rho -> U rho U^dagger on the full matrix, the reference's own test
    oracle (test/utility/linalg.c:27-78, zumu);
  * kraus_to_superop and the superoperator block update (src/channel/channel.c:21-50,
    src/channel/channel_packed.c:8-120);
  * mean / matel_diag (src/meas/meas_pure.c:20-46, meas_packed.c, meas_tiled.c);
  * exp_diag (src/circ/circ_pure.c:21-33; circ_packed.c:28-71 product identity).

Pinning: tests/test_oracle_pin.py checks every function here against the reference library
compiled from its own sources (oracle/_ref, built by oracle/Makefile) over all gates, all
qubit tuples, the reference test fixtures' families and the 12 q / 8 q random-circuit
configuration, and against the known-answer values of the reference test suite.
"""
from __future__ import annotations

import functools

import numpy as np

SQRT1_2 = 0.70710678118654752440  # M_SQRT1_2

GATES_1Q = ("x", "y", "z", "h", "s", "sdg", "t", "tdg", "hy")
GATES_ROT = ("rx", "ry", "rz", "p")
GATES_2Q = ("cx", "cy", "cz", "swap")
GATES_3Q = ("ccx",)
ALL_GATES = GATES_1Q + GATES_ROT + GATES_2Q + GATES_3Q


def arity(name: str) -> int:
    if name in GATES_2Q:
        return 2
    if name in GATES_3Q:
        return 3
    return 1


# ----------------------------------------------------------------------------------------
# storage layouts
# ----------------------------------------------------------------------------------------
def packed_len(n: int) -> int:
    d = 1 << n
    return 1 if n == 0 else (d // 2) * (d + 1)


def tiled_len(n: int, log_tile: int) -> int:
    d, t = 1 << n, 1 << log_tile
    nt = (d + t - 1) // t
    return nt * (nt + 1) // 2 * t * t


def state_len(kind: str, n: int, log_tile: int = 5) -> int:
    if kind == "pure":
        return 1 << n
    if kind == "packed":
        return packed_len(n)
    return tiled_len(n, log_tile)


@functools.lru_cache(maxsize=64)
def _packed_rc(n: int):
    """(row, col) of every packed storage index: column-major lower triangle."""
    col, row = np.triu_indices(1 << n)
    return row.astype(np.int64), col.astype(np.int64)


@functools.lru_cache(maxsize=64)
def _tiled_rc(n: int, log_tile: int):
    """(row, col, live) of every tiled storage index (live False on the padding)."""
    d, t = 1 << n, 1 << log_tile
    idx = np.arange(tiled_len(n, log_tile), dtype=np.int64)
    tile = idx >> (2 * log_tile)
    lr = (idx >> log_tile) & (t - 1)
    lc = idx & (t - 1)
    tr = ((np.sqrt(8.0 * tile + 1.0) - 1.0) // 2).astype(np.int64)
    tr = np.where(tr * (tr + 1) // 2 > tile, tr - 1, tr)
    tr = np.where((tr + 1) * (tr + 2) // 2 <= tile, tr + 1, tr)
    tc = tile - tr * (tr + 1) // 2
    r = tr * t + lr
    c = tc * t + lc
    live = (r < d) & (c < d)
    return r, c, live


def to_storage(kind: str, full: np.ndarray, log_tile: int = 5) -> np.ndarray:
    """Storage array of a full (Hermitian) matrix, or of a vector for PURE."""
    if kind == "pure":
        return np.ascontiguousarray(full, dtype=np.complex128)
    n = int(full.shape[0]).bit_length() - 1
    if kind == "packed":
        r, c = _packed_rc(n)
        return full[r, c].astype(np.complex128)
    r, c, live = _tiled_rc(n, log_tile)
    out = np.zeros(r.shape[0], dtype=np.complex128)
    out[live] = full[r[live], c[live]]
    return out


def from_storage(kind: str, arr: np.ndarray, n: int, log_tile: int = 5) -> np.ndarray:
    """Full matrix (or vector) from storage, reading only the lower triangle."""
    if kind == "pure":
        return np.array(arr, dtype=np.complex128)
    d = 1 << n
    full = np.zeros((d, d), dtype=np.complex128)
    if kind == "packed":
        r, c = _packed_rc(n)
        v = arr
    else:
        r, c, live = _tiled_rc(n, log_tile)
        keep = live & (r >= c)
        r, c, v = r[keep], c[keep], arr[keep]
    full[c, r] = np.conj(v)
    full[r, c] = v
    return full


# ----------------------------------------------------------------------------------------
# gate matrices (reference test/utility/gatemat.c, test/include/test_gate.h)
# ----------------------------------------------------------------------------------------
def gate_matrix(name: str, theta: float | None = None) -> np.ndarray:
    s2 = SQRT1_2
    if name == "x":
        return np.array([[0, 1], [1, 0]], dtype=complex)
    if name == "y":
        return np.array([[0, -1j], [1j, 0]], dtype=complex)
    if name == "z":
        return np.diag([1, -1]).astype(complex)
    if name == "h":
        return np.array([[s2, s2], [s2, -s2]], dtype=complex)
    if name == "hy":
        return np.array([[s2, -s2], [s2, s2]], dtype=complex)
    if name == "s":
        return np.diag([1, 1j])
    if name == "sdg":
        return np.diag([1, -1j])
    if name == "t":
        return np.diag([1, s2 + 1j * s2])
    if name == "tdg":
        return np.diag([1, s2 - 1j * s2])
    if name in ("rx", "ry", "rz"):
        c, s = np.cos(theta / 2.0), np.sin(theta / 2.0)
        if name == "rx":
            return np.array([[c, -1j * s], [-1j * s, c]])
        if name == "ry":
            return np.array([[c, -s], [s, c]], dtype=complex)
        return np.diag([c - 1j * s, c + 1j * s])
    if name == "p":
        return np.diag([1, np.cos(theta) + 1j * np.sin(theta)])
    if name == "cx":
        m = np.eye(4, dtype=complex)
        m[[2, 3]] = m[[3, 2]]
        return m
    if name == "cy":
        m = np.eye(4, dtype=complex)
        m[2, 2] = m[3, 3] = 0
        m[2, 3], m[3, 2] = -1j, 1j
        return m
    if name == "cz":
        return np.diag([1, 1, 1, -1]).astype(complex)
    if name == "swap":
        m = np.eye(4, dtype=complex)
        m[[1, 2]] = m[[2, 1]]
        return m
    if name == "ccx":
        m = np.eye(8, dtype=complex)
        m[[6, 7]] = m[[7, 6]]
        return m
    raise ValueError(name)


def apply_left(m: np.ndarray, u: np.ndarray, qubits, n: int) -> np.ndarray:
    """u applied to the row index of m (a vector or a d x k matrix); qubits[0] = local MSB."""
    k = len(qubits)
    rest = m.shape[1:]
    t = m.reshape([2] * n + list(rest))
    axes = [n - 1 - q for q in qubits]
    t = np.moveaxis(t, axes, list(range(k)))
    shp = t.shape
    t = (u @ t.reshape(1 << k, -1)).reshape(shp)
    t = np.moveaxis(t, list(range(k)), axes)
    return np.ascontiguousarray(t).reshape(m.shape)


def conjugate_by(rho: np.ndarray, u: np.ndarray, qubits, n: int) -> np.ndarray:
    """rho -> U rho U^dagger (reference test oracle zumu, test/utility/linalg.c:44-78)."""
    x = apply_left(rho, u, qubits, n)
    return apply_left(x.T, np.conj(u), qubits, n).T


# ----------------------------------------------------------------------------------------
# PURE gates with the reference pair formulas (src/gate/gate_pure.c)
# ----------------------------------------------------------------------------------------
def _pairs(psi: np.ndarray, q: int):
    v = psi.reshape(-1, 2, 1 << q)
    return v[:, 0, :], v[:, 1, :]


def _cplx(re, im):
    return re + 1j * im


def apply_pure(psi: np.ndarray, name: str, qubits, theta: float | None = None) -> np.ndarray:
    psi = np.array(psi, dtype=np.complex128)
    n = int(psi.shape[0]).bit_length() - 1
    if arity(name) == 1:
        q = qubits[0]
        a, b = _pairs(psi, q)
        a0, b0 = a.copy(), b.copy()
        ar, ai, br, bi = a0.real, a0.imag, b0.real, b0.imag
        if name == "x":
            a[...], b[...] = b0, a0
        elif name == "y":
            a[...], b[...] = _cplx(bi, -br), _cplx(-ai, ar)
        elif name == "z":
            b[...] = -b0
        elif name == "h":
            a[...], b[...] = (a0 + b0) * SQRT1_2, (a0 - b0) * SQRT1_2
        elif name == "hy":
            a[...], b[...] = (a0 - b0) * SQRT1_2, (a0 + b0) * SQRT1_2
        elif name == "s":
            b[...] = _cplx(-bi, br)
        elif name == "sdg":
            b[...] = _cplx(bi, -br)
        elif name == "t":
            b[...] = _cplx((br - bi) * SQRT1_2, (br + bi) * SQRT1_2)
        elif name == "tdg":
            b[...] = _cplx((br + bi) * SQRT1_2, (bi - br) * SQRT1_2)
        elif name == "p":
            c, s = np.cos(theta), np.sin(theta)
            b[...] = _cplx(c * br - s * bi, s * br + c * bi)
        else:
            c, s = np.cos(theta / 2.0), np.sin(theta / 2.0)
            if name == "rx":
                a[...] = c * a0 + _cplx(s * bi, -s * br)
                b[...] = _cplx(s * ai, -s * ar) + c * b0
            elif name == "ry":
                a[...] = c * a0 - s * b0
                b[...] = s * a0 + c * b0
            elif name == "rz":
                a[...] = _cplx(c * ar + s * ai, c * ai - s * ar)
                b[...] = _cplx(c * br - s * bi, c * bi + s * br)
            else:
                raise ValueError(name)
        return psi
    # 2- and 3-qubit gates are permutations with phases: exact index arithmetic
    idx = np.arange(1 << n, dtype=np.int64)
    out = psi.copy()
    if name in ("cx", "cy", "cz"):
        c_, t_ = qubits
        sel = ((idx >> c_) & 1) == 1
        sel0 = sel & (((idx >> t_) & 1) == 0)
        i0 = idx[sel0]
        i1 = i0 | (1 << t_)
        a0, b0 = psi[i0], psi[i1]
        if name == "cx":
            out[i0], out[i1] = b0, a0
        elif name == "cy":
            out[i0], out[i1] = _cplx(b0.imag, -b0.real), _cplx(-a0.imag, a0.real)
        else:
            out[i1] = -b0
        return out
    if name == "swap":
        q1, q2 = qubits
        sel = (((idx >> q1) & 1) == 1) & (((idx >> q2) & 1) == 0)
        i01 = idx[sel]
        i10 = (i01 & ~(1 << q1)) | (1 << q2)
        out[i01], out[i10] = psi[i10], psi[i01]
        return out
    if name == "ccx":
        c1, c2, t_ = qubits
        sel = (((idx >> c1) & 1) == 1) & (((idx >> c2) & 1) == 1) & (((idx >> t_) & 1) == 0)
        i0 = idx[sel]
        i1 = i0 | (1 << t_)
        out[i0], out[i1] = psi[i1], psi[i0]
        return out
    raise ValueError(name)


def apply_mixed(rho: np.ndarray, name: str, qubits, theta: float | None = None) -> np.ndarray:
    n = int(rho.shape[0]).bit_length() - 1
    return conjugate_by(rho, gate_matrix(name, theta), list(qubits), n)


def apply_gate(kind: str, data: np.ndarray, name: str, qubits, theta: float | None = None) -> np.ndarray:
    """Apply a gate to a full vector (pure) or full matrix (mixed)."""
    if kind == "pure":
        return apply_pure(data, name, qubits, theta)
    return apply_mixed(data, name, qubits, theta)


# ----------------------------------------------------------------------------------------
# channels (src/channel/channel.c:21-50, channel_packed.c:8-46)
# ----------------------------------------------------------------------------------------
def kraus_to_superop(kraus) -> np.ndarray:
    """S[(i*N+j), (k*N+l)] = sum_a K_a[i,k] conj(K_a[j,l]) for row-major K_a (N x N)."""
    kraus = [np.asarray(k, dtype=np.complex128) for k in kraus]
    nn = kraus[0].shape[0]
    s = np.zeros((nn * nn, nn * nn), dtype=np.complex128)
    for k in kraus:
        s += np.einsum("ik,jl->ijkl", k, np.conj(k)).reshape(nn * nn, nn * nn)
    return s


def apply_superop1(rho: np.ndarray, sop: np.ndarray, q: int) -> np.ndarray:
    """vec(rho_2x2)' = S vec(rho_2x2) for every 2x2 block of qubit q, vec = (00, 01, 10, 11)."""
    n = int(rho.shape[0]).bit_length() - 1
    t = rho.reshape([2] * (2 * n))
    ra, ca = n - 1 - q, 2 * n - 1 - q
    t = np.moveaxis(t, [ra, ca], [0, 1])
    shp = t.shape
    t = (sop @ t.reshape(4, -1)).reshape(shp)
    t = np.moveaxis(t, [0, 1], [ra, ca])
    return np.ascontiguousarray(t).reshape(rho.shape)


def apply_superop2(rho: np.ndarray, sop: np.ndarray, q0: int, q1: int) -> np.ndarray:
    """vec(rho_4x4)' = S vec(rho_4x4) for every 4x4 block of qubits (q0, q1): vec index
    4 * row + column, local index 2 * bit(q0) + bit(q1).  The library's own 2-qubit channel
    (no reference counterpart; kraus_to_superop builds the 16 x 16 superoperator,
    src/channel/channel.c:21-50), checked against the Kraus sum in the tests."""
    n = int(rho.shape[0]).bit_length() - 1
    t = rho.reshape([2] * (2 * n))
    axes = [n - 1 - q0, n - 1 - q1, 2 * n - 1 - q0, 2 * n - 1 - q1]
    t = np.moveaxis(t, axes, [0, 1, 2, 3])
    shp = t.shape
    t = (sop @ t.reshape(16, -1)).reshape(shp)
    t = np.moveaxis(t, [0, 1, 2, 3], axes)
    return np.ascontiguousarray(t).reshape(rho.shape)


def depolarizing_kraus(p: float):
    """p/4 form of the reference tests (test/channel/test_channel_tiled.c:38-45)."""
    a, b = np.sqrt(1.0 - 3.0 * p / 4.0), np.sqrt(p / 4.0)
    return [a * np.eye(2), b * np.array([[0, 1], [1, 0]]), b * np.array([[0, -1j], [1j, 0]]),
            b * np.array([[1, 0], [0, -1]])]


def amplitude_damping_kraus(gamma: float):
    """test/channel/test_channel_tiled.c:47-53."""
    return [np.array([[1, 0], [0, np.sqrt(1.0 - gamma)]]), np.array([[0, np.sqrt(gamma)], [0, 0]])]


def phase_damping_kraus(lam: float):
    return [np.array([[1, 0], [0, np.sqrt(1.0 - lam)]]), np.array([[0, 0], [0, np.sqrt(lam)]])]


def bitflip_kraus(p: float):
    return [np.sqrt(1 - p) * np.eye(2), np.sqrt(p) * np.array([[0, 1], [1, 0]])]


def phaseflip_kraus(p: float):
    return [np.sqrt(1 - p) * np.eye(2), np.sqrt(p) * np.array([[1, 0], [0, -1]])]


# ----------------------------------------------------------------------------------------
# measurement and diagonal evolution
# ----------------------------------------------------------------------------------------
def mean(kind: str, data: np.ndarray, obs: np.ndarray) -> float:
    if kind == "pure":
        return float(np.sum(obs * (data.real ** 2 + data.imag ** 2)))
    return float(np.sum(obs * np.real(np.diag(data))))


def matel_diag(bra: np.ndarray, ket: np.ndarray, obs: np.ndarray) -> complex:
    re = np.sum(obs * (bra.real * ket.real + bra.imag * ket.imag))
    im = np.sum(obs * (bra.real * ket.imag - bra.imag * ket.real))
    return complex(re, im)


def exp_diag(kind: str, data: np.ndarray, diag: np.ndarray, t: float) -> np.ndarray:
    if t == 0.0:
        return np.array(data, copy=True)
    ang = diag * t
    c, s = np.cos(ang), np.sin(ang)
    if kind == "pure":
        re, im = data.real, data.imag
        return (c * re + s * im) + 1j * (c * im - s * re)
    # e^{-i(d_r - d_c)t} = (c_r - i s_r)(c_c + i s_c)
    f_re = np.outer(c, c) + np.outer(s, s)
    f_im = -np.outer(s, c) + np.outer(c, s)
    re, im = data.real, data.imag
    out = (f_re * re - f_im * im) + 1j * (f_re * im + f_im * re)
    np.fill_diagonal(out, np.diag(data))
    return out


def plus_state(kind: str, n: int) -> np.ndarray:
    d = 1 << n
    if kind == "pure":
        return np.full(d, 1.0 / np.sqrt(float(d)), dtype=np.complex128)
    return np.full((d, d), 1.0 / d, dtype=np.complex128)


# ----------------------------------------------------------------------------------------
# QAOA-style circuits as compositions of reference calls (the batched entry point's checker)
# ----------------------------------------------------------------------------------------
def maxcut_cost(n: int, edges, weights=None) -> np.ndarray:
    """cost[x] = sum_e w_e [bit u_e of x != bit v_e of x], summed in edge order (unit
    weights: counted in small integers, the same values)."""
    if weights is None:
        x = np.arange(1 << n, dtype=np.uint32)
        cnt = np.zeros(1 << n, dtype=np.uint8 if len(edges) < 256 else np.uint32)
        for u, v in edges:
            np.add(cnt, ((x >> u) ^ (x >> v)) & 1, out=cnt, casting="unsafe")
        return cnt.astype(np.float64)
    x = np.arange(1 << n, dtype=np.int64)
    cost = np.zeros(1 << n, dtype=np.float64)
    for e, (u, v) in enumerate(edges):
        w = 1.0 if weights is None else float(weights[e])
        cost += w * (((x >> u) ^ (x >> v)) & 1)
    return cost


def qaoa_state(n: int, cost: np.ndarray, gammas, betas, low_qubits: int | None = None,
               layers: int | None = None, last_half: str | None = None) -> np.ndarray:
    """state_plus (src/state/state_pure.c:30-43), then per layer k: exp_diag(cost, gamma_k)
    (src/circ/circ_pure.c:21-33) and rx(q, 2 beta_k) on every qubit (src/gate/gate_pure.c:
    230-234).  `layers` stops after that many layers; `last_half` = "low" / "high" applies
    only the rx on qubits < low_qubits / >= low_qubits in the last layer."""
    psi = plus_state("pure", n)
    nl = len(gammas) if layers is None else layers
    for k in range(nl):
        psi = exp_diag("pure", psi, cost, float(gammas[k]))
        qs = range(n)
        if k == nl - 1 and last_half is not None:
            qs = range(low_qubits) if last_half == "low" else range(low_qubits, n)
        for q in qs:
            psi = apply_pure(psi, "rx", [q], 2.0 * float(betas[k]))
    return psi


def qaoa_mean(n: int, cost: np.ndarray, gammas, betas) -> float:
    """mean(cost) of the QAOA state (src/meas/meas_pure.c:20-30)."""
    return mean("pure", qaoa_state(n, cost, gammas, betas), cost)
