"""Seeded synthetic workloads of the benchmark configurations (no datasets involved).

* random circuits: gates uniform over the 18 gate calls, distinct qubits uniform,
  rotation angles uniform in [0, 2 pi) (the 12 q PURE / 8 q mixed parity configuration);
* Gaussian-random normalised pure states and Dirichlet(1,1,1,1)-weighted mixtures of 4
  such states (the 30 q / 14 q / 13 q throughput configurations);
* the single-gate throughput sweep: every 1-qubit gate on every target, 2-qubit gates on
  (low, high), (high, low) and adjacent pairs, CCX on adjacent and spread triples.

All generators use numpy's PCG64 stream with an explicit seed.
"""
from __future__ import annotations

import math

import numpy as np

GATES_1Q = ("x", "y", "z", "h", "s", "sdg", "t", "tdg", "hy")
GATES_ROT = ("rx", "ry", "rz", "p")
GATES_2Q = ("cx", "cy", "cz", "swap")
ALL_GATES = GATES_1Q + GATES_ROT + GATES_2Q + ("ccx",)


def gate_arity(name: str) -> int:
    return 2 if name in GATES_2Q else (3 if name == "ccx" else 1)


def random_circuit(n: int, n_gates: int, seed: int):
    """[(name, qubits, theta or None)] with gates uniform over the 18 calls."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_gates):
        name = ALL_GATES[int(rng.integers(len(ALL_GATES)))]
        k = gate_arity(name)
        qs = tuple(int(q) for q in rng.choice(n, size=k, replace=False))
        theta = float(rng.uniform(0.0, 2.0 * math.pi)) if name in GATES_ROT else None
        out.append((name, qs, theta))
    return out


def gaussian_pure(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return v / np.linalg.norm(v)


def dirichlet_mixture_terms(n: int, seed: int, k: int = 4):
    """Weights w ~ Dirichlet(1,...,1) and k Gaussian normalised pure states psi_i."""
    rng = np.random.default_rng(seed)
    w = rng.dirichlet(np.ones(k))
    psis = []
    for _ in range(k):
        v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
        psis.append(v / np.linalg.norm(v))
    return w, psis


def dirichlet_mixture(n: int, seed: int, k: int = 4) -> np.ndarray:
    """Full matrix rho = sum_i w_i |psi_i><psi_i| (small n only)."""
    w, psis = dirichlet_mixture_terms(n, seed, k)
    rho = np.zeros((1 << n, 1 << n), dtype=np.complex128)
    for wi, p in zip(w, psis):
        rho += wi * np.outer(p, np.conj(p))
    return rho


def uniform_obs(n: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).uniform(-1.0, 1.0, size=1 << n)


def sweep(n: int):
    """The single-gate throughput sweep on n qubits: [(name, qubits, theta)]."""
    rng = np.random.default_rng(1234 + n)
    out = []
    for name in GATES_1Q + GATES_ROT:
        for q in range(n):
            theta = float(rng.uniform(0.0, 2.0 * math.pi)) if name in GATES_ROT else None
            out.append((name, (q,), theta))
    lo, hi = 0, n - 1
    pairs = [(lo, hi), (hi, lo)] + [(q, q + 1) for q in range(n - 1)]
    for name in GATES_2Q:
        for pr in pairs:
            out.append((name, pr, None))
    triples = [(0, n // 2, n - 1), (n - 1, n // 2, 0)] + [(q, q + 1, q + 2) for q in range(n - 2)]
    for tr in triples:
        out.append(("ccx", tr, None))
    return out


def channel_set(n: int, seed: int):
    """The Kraus-channel throughput configuration on n qubits: on every qubit a depolarizing
    channel (p ~ U[0, 0.1], p/4 form), amplitude damping (gamma ~ U[0, 0.2]), phase damping
    (lambda ~ U[0, 0.2]) and a random 4-operator CPTP channel (the 2 x 2 blocks of the QR
    isometry of a Gaussian complex 8 x 2 matrix).  Returns [(label, kraus, qubit)]."""
    rng = np.random.default_rng(4321 + n)
    out = []
    x = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    y = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
    z = np.array([[1, 0], [0, -1]], dtype=np.complex128)
    for q in range(n):
        p = rng.uniform(0.0, 0.1)
        a, b = math.sqrt(1.0 - 3.0 * p / 4.0), math.sqrt(p / 4.0)
        out.append(("depolarizing", [a * np.eye(2), b * x, b * y, b * z], q))
        g = rng.uniform(0.0, 0.2)
        out.append(("amplitude_damping", [np.array([[1, 0], [0, math.sqrt(1 - g)]], dtype=np.complex128),
                                          np.array([[0, math.sqrt(g)], [0, 0]], dtype=np.complex128)], q))
        lam = rng.uniform(0.0, 0.2)
        out.append(("phase_damping", [np.array([[1, 0], [0, math.sqrt(1 - lam)]], dtype=np.complex128),
                                      np.array([[0, 0], [0, math.sqrt(lam)]], dtype=np.complex128)], q))
        iso, _ = np.linalg.qr(rng.standard_normal((8, 2)) + 1j * rng.standard_normal((8, 2)))
        out.append(("random_cptp", [iso[2 * i:2 * i + 2, :] for i in range(4)], q))
    return out


# ---------------------------------------------------------------------------------------
# device-side generation of the large benchmark states (torch is only the RNG/plumbing)
# ---------------------------------------------------------------------------------------
class _DeviceArray:
    """Zero-copy view of library-owned device memory for torch (__cuda_array_interface__)."""

    def __init__(self, ptr: int, count: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def state_view(ork, st):
    """torch complex128 tensor aliasing a state's device storage (queued statevector gates
    are launched first, so the view sees every gate applied so far)."""
    import ctypes as C

    import torch
    ork.lib.orkan_flush()
    count = int(ork.lib.state_len(C.byref(st)))
    return torch.as_tensor(_DeviceArray(int(st.data), count, "<c16"), device="cuda")


def storage_rc_torch(kind: str, n: int, log_tile: int, device="cuda"):
    """(row, col, live) of every storage index, on the device."""
    import torch
    d = 1 << n
    if kind == "packed":
        idx = torch.triu_indices(d, d, device=device)
        return idx[1], idx[0], None
    t = 1 << log_tile
    nt = (d + t - 1) // t
    e = torch.arange(nt * (nt + 1) // 2 * t * t, device=device, dtype=torch.int64)
    tile = e >> (2 * log_tile)
    lr = (e >> log_tile) & (t - 1)
    lc = e & (t - 1)
    tr = torch.floor((torch.sqrt(8.0 * tile.double() + 1.0) - 1.0) / 2).long()
    tr = torch.where(tr * (tr + 1) // 2 > tile, tr - 1, tr)
    tr = torch.where((tr + 1) * (tr + 2) // 2 <= tile, tr + 1, tr)
    tc = tile - tr * (tr + 1) // 2
    r, c = tr * t + lr, tc * t + lc
    return r, c, (r < d) & (c < d)


def initial_storage_torch(kind: str, n: int, seed: int, log_tile: int = 5, device="cuda"):
    """Storage of the benchmark's initial state: a Gaussian normalised statevector, or a
    Dirichlet(1,1,1,1) mixture of 4 Gaussian normalised states in the given layout."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    d = 1 << n

    def gauss():
        v = torch.complex(torch.randn(d, generator=g, device=device, dtype=torch.float64),
                          torch.randn(d, generator=g, device=device, dtype=torch.float64))
        return v / torch.linalg.vector_norm(v)

    if kind == "pure":
        return gauss()
    w = np.random.default_rng(seed).dirichlet(np.ones(4))
    r, c, live = storage_rc_torch(kind, n, log_tile, device)
    out = torch.zeros(r.shape[0], dtype=torch.complex128, device=device)
    for wi in w:
        p = gauss()
        term = p[r.clamp(max=d - 1)] * torch.conj(p[c.clamp(max=d - 1)])
        out += float(wi) * (term if live is None else torch.where(live, term, torch.zeros_like(term)))
        del term, p
    return out


def initial_storage(kind: str, n: int, seed: int, log_tile: int = 5) -> np.ndarray:
    """Host copy of initial_storage_torch (generated on the GPU when one is present)."""
    try:
        import torch
        if torch.cuda.is_available():
            return initial_storage_torch(kind, n, seed, log_tile).cpu().numpy()
        return initial_storage_torch(kind, n, seed, log_tile, device="cpu").numpy()
    except ImportError:
        raise RuntimeError("torch is needed to generate the benchmark states")


def fill_state_on_device(ork, st, kind: str, n: int, seed: int, log_tile: int = 5) -> None:
    import torch
    state_view(ork, st).copy_(initial_storage_torch(kind, n, seed, log_tile))
    torch.cuda.synchronize()


def uniform_obs_torch(n: int, seed: int):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.rand(1 << n, generator=g, device="cuda", dtype=torch.float64) * 2.0 - 1.0
