"""Binding of the batched QAOA entry points (include/orkan_batch.h) in liborkan_b200.so.

    b = QaoaBatch(ork, n_list, edges_list, weights_list, p)
    means = b.run(gammas, betas)          # [count][p] angles in instance order -> [count] means
    b.tune(gammas, betas, cache_path)     # autotune chunk and block size per qubit count
    b.close()

Every call goes to the compiled library; there is no Python fallback.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import OrkanError


def _declare(lib):
    if getattr(lib, "_qaoa_declared", False):
        return
    P = C.c_void_p
    lib.orkan_qaoa_create.argtypes = [C.POINTER(P), C.c_uint, P, P, P, P, C.c_uint, C.c_ulonglong, C.c_uint]
    lib.orkan_qaoa_run.argtypes = [P, P, P, P, P]
    lib.orkan_qaoa_tune.argtypes = [P, P, P, C.c_char_p]
    lib.orkan_qaoa_config.argtypes = [P, C.c_uint, C.POINTER(C.c_uint), C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
    lib.orkan_qaoa_cost_vector.argtypes = [P, C.c_uint, P]
    lib.orkan_qaoa_stats.argtypes = [P, C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
    lib.orkan_qaoa_destroy.argtypes = [P]
    lib.orkan_qaoa_destroy.restype = None
    for f in ("create", "run", "tune", "config", "cost_vector", "stats"):
        getattr(lib, "orkan_qaoa_" + f).restype = C.c_int
    lib._qaoa_declared = True


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise OrkanError(f"orkan_qaoa_{what} failed with CUDA error {rc}")


class QaoaBatch:
    """count instances of MaxCut-cost QAOA circuits with a shared depth p."""

    def __init__(self, ork, n_qubits, edges, weights=None, p: int = 1, mem_budget: int = 0,
                 f64_costs: bool = False):
        self.lib = ork.lib
        _declare(self.lib)
        self.n = np.ascontiguousarray(n_qubits, dtype=np.uint32)
        self.count, self.p = len(self.n), int(p)
        off = np.zeros(self.count + 1, dtype=np.uint32)
        flat = []
        wflat = []
        for i, es in enumerate(edges):
            off[i + 1] = off[i] + len(es)
            flat.extend(int(v) for e in es for v in e)
            if weights is not None:
                wflat.extend(float(x) for x in weights[i])
        self._off = off
        self._edges = np.ascontiguousarray(flat if flat else [0], dtype=np.uint32)
        self._w = np.ascontiguousarray(wflat, dtype=np.float64) if weights is not None else None
        h = C.c_void_p()
        rc = self.lib.orkan_qaoa_create(C.byref(h), self.count, self.n.ctypes.data, off.ctypes.data,
                                        self._edges.ctypes.data,
                                        None if self._w is None else self._w.ctypes.data, self.p,
                                        int(mem_budget), 1 if f64_costs else 0)
        _check(rc, "create")
        self.h = h

    def _angles(self, gammas, betas):
        g = np.ascontiguousarray(gammas, dtype=np.float64).reshape(self.count, self.p)
        b = np.ascontiguousarray(betas, dtype=np.float64).reshape(self.count, self.p)
        return g, b

    def run(self, gammas, betas, stream: int | None = None) -> np.ndarray:
        g, b = self._angles(gammas, betas)
        out = np.empty(self.count, dtype=np.float64)
        _check(self.lib.orkan_qaoa_run(self.h, g.ctypes.data, b.ctypes.data, out.ctypes.data, stream), "run")
        return out

    def tune(self, gammas, betas, cache_path: str | None = None) -> None:
        g, b = self._angles(gammas, betas)
        path = None if cache_path is None else cache_path.encode()
        _check(self.lib.orkan_qaoa_tune(self.h, g.ctypes.data, b.ctypes.data, path), "tune")

    def config(self, n: int) -> tuple[int, int, int]:
        """(log2 chunk, threads per block, shared buffers per block) for n-qubit instances."""
        lc, t, r = C.c_uint(), C.c_uint(), C.c_uint()
        _check(self.lib.orkan_qaoa_config(self.h, n, C.byref(lc), C.byref(t), C.byref(r)), "config")
        return lc.value, t.value, r.value

    def cost_vector(self, i: int) -> np.ndarray:
        out = np.empty(1 << int(self.n[i]), dtype=np.float64)
        _check(self.lib.orkan_qaoa_cost_vector(self.h, i, out.ctypes.data), "cost_vector")
        return out

    def stats(self) -> tuple[int, int]:
        w, l = C.c_uint(), C.c_uint()
        _check(self.lib.orkan_qaoa_stats(self.h, C.byref(w), C.byref(l)), "stats")
        return w.value, l.value

    def close(self) -> None:
        if self.h:
            self.lib.orkan_qaoa_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def shard_instances(n_qubits, world: int) -> list[np.ndarray]:
    """Partition instances over `world` ranks by work (2^n amplitude-passes each): instances
    in descending order of n (index order among equals), each to the rank with the least
    work so far (lowest rank on ties).  Returns each rank's instance indices, ascending.
    Deterministic, so every rank computes the same partition without communication."""
    n = np.asarray(n_qubits, dtype=np.int64)
    if world < 1:
        raise ValueError("world must be at least 1")
    order = sorted(range(len(n)), key=lambda i: (-int(n[i]), i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += 1 << int(n[i])
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def scatter_means(count: int, idx, local_means) -> np.ndarray:
    """A full-length vector holding this rank's means at their instance indices and 0.0
    elsewhere; the sum of all ranks' vectors is the whole batch (x + 0.0 == x exactly)."""
    out = np.zeros(count, dtype=np.float64)
    if len(idx):
        out[np.asarray(idx)] = np.asarray(local_means, dtype=np.float64)
    return out


def gather_means(count: int, idx, local_means, dist=None, device="cpu") -> np.ndarray:
    """Every rank's means in instance order, on every rank (one all-reduce of `count`
    doubles over the process group; the local vector alone without one)."""
    part = scatter_means(count, idx, local_means)
    if dist is None:
        return part
    import torch
    t = torch.from_numpy(part).to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy()


class ShardedQaoaBatch:
    """This rank's share of a QAOA batch spread over `world` ranks (one GPU each): the
    instances of `shard_instances(n_qubits, world)[rank]` in a local QaoaBatch.  `run`
    evaluates the local share; `gather` assembles the whole batch's means on every rank.
    Instances are independent, so the only exchange is that final gather."""

    def __init__(self, ork, n_qubits, edges, weights=None, p: int = 1, rank: int = 0, world: int = 1, **kw):
        self.count, self.p = len(n_qubits), int(p)
        self.idx = shard_instances(n_qubits, world)[rank]
        sel = [int(i) for i in self.idx]
        self.local = None
        if sel:
            self.local = QaoaBatch(ork, [int(n_qubits[i]) for i in sel], [edges[i] for i in sel],
                                   None if weights is None else [weights[i] for i in sel], p, **kw)

    def _local_angles(self, gammas, betas):
        g = np.asarray(gammas, dtype=np.float64).reshape(self.count, self.p)[self.idx]
        b = np.asarray(betas, dtype=np.float64).reshape(self.count, self.p)[self.idx]
        return g, b

    def tune(self, gammas, betas, cache_path: str | None = None) -> None:
        if self.local is not None:
            self.local.tune(*self._local_angles(gammas, betas), cache_path)

    def run(self, gammas, betas) -> np.ndarray:
        """Means of this rank's instances (in the order of `self.idx`)."""
        if self.local is None:
            return np.zeros(0)
        return self.local.run(*self._local_angles(gammas, betas))

    def gather(self, local_means, dist=None, device="cpu") -> np.ndarray:
        return gather_means(self.count, self.idx, local_means, dist, device)

    def close(self) -> None:
        if self.local is not None:
            self.local.close()
            self.local = None


def random_regular_graph(n: int, d: int, rng) -> list[tuple[int, int]]:
    """A uniformly drawn simple d-regular graph on n vertices (configuration model with
    rejection of loops and multi-edges).  When n * d is odd no such graph exists; then one
    random vertex gets degree d - 1 and all others degree d."""
    if d >= n:
        raise ValueError("degree must be below the vertex count")
    deg = np.full(n, d)
    if (n * d) % 2:
        deg[rng.integers(n)] -= 1
    while True:
        stubs = rng.permutation(np.repeat(np.arange(n), deg))
        pairs = stubs.reshape(-1, 2)
        if np.any(pairs[:, 0] == pairs[:, 1]):
            continue
        key = {tuple(sorted(map(int, e))) for e in pairs}
        if len(key) == len(pairs):
            return [tuple(int(v) for v in e) for e in pairs]


def erdos_renyi_graph(n: int, prob: float, rng) -> list[tuple[int, int]]:
    return [(u, v) for u in range(n) for v in range(u + 1, n) if rng.random() < prob]


def _main(argv=None):
    """Run one batch of 3-regular MaxCut instances: python -m orkan_b200.batch --count 64
    --qubits 20 [--p 4 --chunk 12 --threads 256 --ring 1 --runs 2].  With --chunk the
    launch configuration of that qubit count is set through a tuner cache file instead of
    tuning.  Prints the configuration, the first mean and the time per run."""
    import argparse
    import json
    import os
    import tempfile
    import time

    import orkan_b200

    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=64)
    ap.add_argument("--qubits", type=int, default=20)
    ap.add_argument("--p", type=int, default=4)
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--threads", type=int, default=256)
    ap.add_argument("--ring", type=int, default=1)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--f64", action="store_true")
    a = ap.parse_args(argv)
    ork = orkan_b200.load(5)
    rng = np.random.default_rng(5)
    edges = [random_regular_graph(a.qubits, 3, rng) for _ in range(a.count)]
    g = rng.uniform(0, np.pi, (a.count, a.p))
    b = rng.uniform(0, np.pi / 2, (a.count, a.p))
    bt = QaoaBatch(ork, [a.qubits] * a.count, edges, None, a.p, f64_costs=a.f64)
    if a.chunk:
        import torch
        key = f"{torch.cuda.get_device_name()}|n{a.qubits}|p{a.p}|{'f64' if a.f64 else 'u8'}|v2"
        fd, path = tempfile.mkstemp(suffix=".json")
        with os.fdopen(fd, "w") as f:
            f.write(json.dumps({key: {"C": a.chunk, "threads": a.threads, "ring": a.ring}}) + "\n")
        bt.tune(g, b, path)
        os.unlink(path)
    means = bt.run(g, b)
    t0 = time.perf_counter()
    for _ in range(a.runs):
        means = bt.run(g, b)
    dt = (time.perf_counter() - t0) / max(1, a.runs)
    print(json.dumps({"config": bt.config(a.qubits), "stats": bt.stats(), "mean0": float(means[0]),
                      "ms_per_run": dt * 1e3}))
    bt.close()


if __name__ == "__main__":
    _main()
