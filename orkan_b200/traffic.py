"""Algorithmic bytes of one gate application (the bandwidth model of the benchmark).

bytes = 2 * 32 B * (number of distinct 32-byte sectors of the storage that hold at least
one element the operation may change).  For operations that change every element this
equals the reference's own convention, 2 x storage bytes (reference docs/BENCHMARK.md
section 6.2, profile/include/profile.h:129-141); for operations that change only part
of the state (Z/S/T/P on a statevector, CZ, controlled gates ...) only the sectors the
operation must read and write are counted, so achieved/peak stays a true fraction.

A sector holds two complex128 elements: storage indices (2k, 2k+1).  "May change" is a
predicate on the bits of the element's row (and column) index at the gate's qubits.
The counts are exact: PURE by enumerating the relevant bit patterns; TILED (sectors
are aligned pairs of columns inside a tile row) by aggregating tiles per high-bit
class; PACKED (sectors follow the storage index, whose parity alignment varies by
column) per column with periodic prefix sums; a sector that straddles two columns is
counted once.
"""
from __future__ import annotations

import functools
import itertools

import numpy as np

DENSE_1Q = ("x", "y", "h", "hy", "rx", "ry")
PHASE_1Q = ("z", "s", "sdg", "t", "tdg", "p", "rz")


def _bit(x, q):
    return (x >> q) & 1


def pure_changes(name, qubits):
    """Predicate over the amplitude index x (numpy int arrays)."""
    if name in DENSE_1Q or name == "rz":
        return lambda x: np.ones_like(x, dtype=bool)
    if name in PHASE_1Q:
        q = qubits[0]
        return lambda x: _bit(x, q) == 1
    if name in ("cx", "cy"):
        c = qubits[0]
        return lambda x: _bit(x, c) == 1
    if name == "cz":
        a, b = qubits
        return lambda x: (_bit(x, a) & _bit(x, b)) == 1
    if name == "swap":
        a, b = qubits
        return lambda x: _bit(x, a) != _bit(x, b)
    if name == "ccx":
        a, b = qubits[0], qubits[1]
        return lambda x: (_bit(x, a) & _bit(x, b)) == 1
    raise ValueError(name)


def mixed_changes(name, qubits):
    """Predicate over (r, c) of the density matrix (numpy int arrays)."""
    if name in DENSE_1Q or name == "channel":
        return lambda r, c: np.ones(np.broadcast(r, c).shape, dtype=bool)
    if name in PHASE_1Q:
        q = qubits[0]
        return lambda r, c: _bit(r, q) != _bit(c, q)
    if name in ("cx", "cy"):
        k = qubits[0]
        return lambda r, c: (_bit(r, k) | _bit(c, k)) == 1
    if name == "cz":
        a, b = qubits
        return lambda r, c: (_bit(r, a) & _bit(r, b)) != (_bit(c, a) & _bit(c, b))
    if name == "swap":
        a, b = qubits
        return lambda r, c: (_bit(r, a) != _bit(r, b)) | (_bit(c, a) != _bit(c, b))
    if name == "ccx":
        a, b = qubits[0], qubits[1]
        return lambda r, c: ((_bit(r, a) & _bit(r, b)) | (_bit(c, a) & _bit(c, b))) == 1
    raise ValueError(name)


def relevant_qubits(name, qubits):
    if name in ("cx", "cy"):
        return (qubits[0],)
    if name == "ccx":
        return (qubits[0], qubits[1])
    if name in DENSE_1Q or name == "channel":
        return ()
    return tuple(qubits)


# ---------------------------------------------------------------------------------------
def pure_sectors(n: int, name: str, qubits) -> int:
    pred = pure_changes(name, qubits)
    if n == 0:
        return 1
    bits = sorted(set(relevant_qubits(name, qubits)) | {0})
    # enumerate the relevant bits; sector = pattern of bits other than bit 0
    touched = 0
    groups = {}
    for pat in itertools.product((0, 1), repeat=len(bits)):
        x = sum(b << q for b, q in zip(pat, bits))
        key = tuple(b for b, q in zip(pat, bits) if q != 0)
        groups[key] = groups.get(key, False) or bool(pred(np.array([x]))[0])
    touched = sum(1 for v in groups.values() if v)
    free_bits = n - len(bits)
    return touched << free_bits


@functools.lru_cache(maxsize=None)
def _tile_pairs(n_tiles: int):
    tr, tc = np.tril_indices(n_tiles)
    return tr.astype(np.int64), tc.astype(np.int64)


def tiled_sectors(n: int, log_tile: int, name: str, qubits) -> int:
    pred = mixed_changes(name, qubits)
    d, t = 1 << n, 1 << log_tile
    if d < t:   # single padded tile, live corner d x d (sectors pair columns 2k, 2k+1)
        r, c = np.meshgrid(np.arange(d), np.arange(0, d, 2), indexing="ij")
        ch = pred(r, c) | pred(r, c + 1) if d > 1 else pred(r, c)
        return int(ch.sum())
    nt = d >> log_tile
    rq = [q for q in relevant_qubits(name, qubits) if q >= log_tile]
    hi = sorted(set(rq))
    tr, tc = _tile_pairs(nt)
    # class of each tile: high bits of tr and tc
    key = np.zeros(tr.shape, dtype=np.int64)
    for j, q in enumerate(hi):
        key |= ((tr >> (q - log_tile)) & 1) << (2 * j)
        key |= ((tc >> (q - log_tile)) & 1) << (2 * j + 1)
    counts = np.bincount(key, minlength=1 << (2 * len(hi)))
    lr, lc = np.meshgrid(np.arange(t), np.arange(0, t, 2), indexing="ij")
    total = 0
    for k, cnt in enumerate(counts):
        if cnt == 0:
            continue
        base_r = sum(((k >> (2 * j)) & 1) << q for j, q in enumerate(hi))
        base_c = sum(((k >> (2 * j + 1)) & 1) << q for j, q in enumerate(hi))
        r = base_r + lr
        c = base_c + lc
        within = int((pred(r, c) | pred(r, c + 1)).sum())
        total += int(cnt) * within
    return total


def packed_sectors(n: int, name: str, qubits) -> int:
    pred = mixed_changes(name, qubits)
    d = 1 << n
    if d == 1:
        return 1
    rel = sorted(set(relevant_qubits(name, qubits)))
    m = max(rel + [1]) + 1
    period = 1 << m            # predicate is periodic in r with this period (for fixed c)
    half = period // 2
    cols = np.arange(d, dtype=np.int64)
    start = cols * (2 * d - cols + 1) // 2        # storage index of (c, c)
    align = (start - cols) & 1                    # rows r with (r - align) even start a sector
    ckey = np.zeros(d, dtype=np.int64)
    for j, q in enumerate(rel):
        ckey |= ((cols >> q) & 1) << j
    cls = ckey * 2 + align
    total = 0
    rr = np.arange(period, dtype=np.int64)
    for k in np.unique(cls):
        sel = np.nonzero(cls == k)[0]
        a = int(k & 1)
        cbits = int(k >> 1)
        c_rep = sum(((cbits >> j) & 1) << q for j, q in enumerate(rel))
        p = pred(rr, np.full_like(rr, c_rep))                       # p(r) over one period
        g = p[(2 * np.arange(half) + a) % period] | p[(2 * np.arange(half) + 1 + a) % period]
        gpre = np.concatenate([[0], np.cumsum(g)])

        def full_pairs(k0, k1):                                       # sum g[k mod half], k in [k0, k1)
            def s(kk):
                return (kk // half) * gpre[half] + gpre[kk % half]
            return s(k1) - s(k0)

        c = sel
        first_partial = ((c - a) & 1) == 1                            # row c pairs with row c - 1
        r0 = np.where(first_partial, c + 1, c)                        # first row of a full pair
        last = d - 1
        last_partial = ((last - a) & 1) == 0                          # row d-1 pairs with row d
        r_end = last if last_partial else d                           # rows [r0, r_end) form full pairs
        k0 = (r0 - a) // 2
        k1 = (r_end - a) // 2
        cnt = full_pairs(k0, np.maximum(k1, k0))
        # a sector straddling columns c-1 and c is counted by column c-1 when its element
        # there (row d-1) changes, else by column c when row c changes
        prev_changed = np.zeros(c.shape, dtype=bool)
        has_prev = c > 0
        prev_changed[has_prev] = pred(np.full(int(has_prev.sum()), d - 1), c[has_prev] - 1)
        cnt = cnt + np.where(first_partial & ~prev_changed, p[c % period], False)
        if last_partial:
            cnt = cnt + p[last % period] * np.ones_like(c)
        total += int(cnt.sum())
    return total


def sectors(kind: str, n: int, name: str, qubits, log_tile: int = 5) -> int:
    if kind == "pure":
        return pure_sectors(n, name, qubits)
    if kind == "packed":
        return packed_sectors(n, name, qubits)
    return tiled_sectors(n, log_tile, name, qubits)


def gate_bytes(kind: str, n: int, name: str, qubits, log_tile: int = 5) -> int:
    """Algorithmic bytes (read + write) of one application."""
    return 2 * 32 * sectors(kind, n, name, qubits, log_tile)


def exp_diag_bytes(kind: str, n: int, log_tile: int = 5) -> int:
    """exp_diag changes every off-diagonal element: 2 x storage bytes plus the 8-byte diag
    entries read once per index."""
    from math import ceil
    d = 1 << n
    if kind == "pure":
        length = d
    elif kind == "packed":
        length = 1 if n == 0 else (d // 2) * (d + 1)
    else:
        t = 1 << log_tile
        nt = (d + t - 1) // t
        length = nt * (nt + 1) // 2 * t * t if d >= t else d * d
    return 2 * 32 * ceil(length / 2) + 8 * d


def mean_bytes(kind: str, n: int) -> int:
    """mean reads |psi|^2 terms (16 B) and obs (8 B) per index; mixed layouts the diagonal."""
    return 24 * (1 << n)
