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
