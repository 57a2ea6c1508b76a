"""CPU oracle of the sample matrix (test infrastructure: only tests import it).

The reference specifies the operation but ships no implementation
(docs/SAMPLE_MATRIX.md: definition in section 1, the brute-force check of section 7).
This is that brute force: every leaf
    |psi_a> = K_{L-1} ... K_{at+1} M_at[a] K_{at-1} ... K_0 |iota>,  K_l = sum_m w_l[m] M_l[m]
is built independently from a copy of |iota> and S[a, b] = <psi_a| diag(obs) |psi_b> is a
plain length-2^n reduction.  Operations are callables on numpy statevectors (returning
the new vector); the gates they apply come from oracle/restate.py, which is pinned to the
reference library.  Parity of the composite is pinned through its parts only: the
reference has no sample matrix to compare against.
"""
from __future__ import annotations

import numpy as np


def apply_channel(ops, weights, psi: np.ndarray) -> np.ndarray:
    out = np.zeros_like(psi)
    for op, w in zip(ops, weights):
        out = out + complex(w) * op(psi.copy())
    return out


def leaves(iota: np.ndarray, channels, at: int) -> list[np.ndarray]:
    vecs = []
    for a, op in enumerate(channels[at][0]):
        psi = iota.astype(np.complex128).copy()
        for l in range(at):
            psi = apply_channel(channels[l][0], channels[l][1], psi)
        psi = op(psi)
        for l in range(at + 1, len(channels)):
            psi = apply_channel(channels[l][0], channels[l][1], psi)
        vecs.append(psi)
    return vecs


def sample_matrix(iota: np.ndarray, obs: np.ndarray, channels, at: int) -> np.ndarray:
    """channels: list of (ops, weights); ops callables psi -> psi'."""
    vecs = leaves(iota, channels, at)
    k = len(vecs)
    s = np.zeros((k, k), dtype=np.complex128)
    for a in range(k):
        for b in range(k):
            s[a, b] = np.sum(np.conj(vecs[a]) * obs * vecs[b])
    return s
