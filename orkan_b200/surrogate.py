"""Binding of the FP32 surrogate network (include/orkan_mlp.h) and the surrogate-guided
angle search built on it and on the batched simulator (include/orkan_batch.h).

    net = Mlp(ork, n_in=12, hidden=256, max_batch=1024, seed=1)
    net.train(x_dev, t_dev, epochs=..., batch=1024, lr=1e-3)     # device tensors (torch)
    y = net.forward(x_dev)
    x_new = net.ascend(x0_dev, steps=200, lr=0.02)                 # proposals

Device memory comes from torch tensors (plumbing only: every computation is a call into
liborkan_b200.so); there is no Python fallback.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import OrkanError


def _declare(lib):
    if getattr(lib, "_mlp_declared", False):
        return
    P = C.c_void_p
    lib.orkan_mlp_create.argtypes = [C.POINTER(P), C.c_uint, C.c_uint, C.c_uint, C.c_ulonglong]
    lib.orkan_mlp_destroy.argtypes = [P]
    lib.orkan_mlp_destroy.restype = None
    lib.orkan_mlp_param_count.argtypes = [P]
    lib.orkan_mlp_param_count.restype = C.c_size_t
    lib.orkan_mlp_get_params.argtypes = [P, P]
    lib.orkan_mlp_set_params.argtypes = [P, P]
    lib.orkan_mlp_forward.argtypes = [P, P, C.c_uint, P, P]
    lib.orkan_mlp_gradients.argtypes = [P, P, P, C.c_uint, P, P, P, P]
    lib.orkan_mlp_train.argtypes = [P, P, P, C.c_uint, C.c_uint, C.c_uint, C.c_float, C.c_ulonglong, P, P]
    lib.orkan_mlp_ascend.argtypes = [P, P, C.c_uint, C.c_uint, C.c_float, C.c_float, C.c_float, P, P]
    lib.orkan_mlp_launch_count.argtypes = []
    lib.orkan_mlp_launch_count.restype = C.c_ulonglong
    for f in ("create", "get_params", "set_params", "forward", "gradients", "train", "ascend"):
        getattr(lib, "orkan_mlp_" + f).restype = C.c_int
    lib._mlp_declared = True


def _check(rc, what):
    if rc != 0:
        raise OrkanError(f"orkan_mlp_{what} failed with CUDA error {rc}")


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class Mlp:
    """12 -> hidden -> hidden -> 1 GELU network with its own CUDA kernels."""

    def __init__(self, ork, n_in=12, hidden=256, max_batch=1024, seed=1):
        self.lib = ork.lib
        _declare(self.lib)
        self.n_in, self.hidden, self.max_batch = n_in, hidden, max_batch
        h = C.c_void_p()
        _check(self.lib.orkan_mlp_create(C.byref(h), n_in, hidden, max_batch, seed), "create")
        self.h = h

    @property
    def param_count(self) -> int:
        return int(self.lib.orkan_mlp_param_count(self.h))

    def get_params(self) -> np.ndarray:
        out = np.empty(self.param_count, dtype=np.float32)
        _check(self.lib.orkan_mlp_get_params(self.h, out.ctypes.data), "get_params")
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.param_count
        _check(self.lib.orkan_mlp_set_params(self.h, p.ctypes.data), "set_params")

    def forward(self, x):
        import torch
        n = x.shape[0]
        y = torch.empty(n, dtype=torch.float32, device=x.device)
        for c0 in range(0, n, self.max_batch):
            c1 = min(n, c0 + self.max_batch)
            xs, ys = x[c0:c1], y[c0:c1]
            _check(self.lib.orkan_mlp_forward(self.h, _ptr(xs), c1 - c0, _ptr(ys), _stream()), "forward")
        return y

    def gradients(self, x, t, want_x=False):
        import torch
        g = torch.empty(self.param_count, dtype=torch.float32, device=x.device)
        gx = torch.empty_like(x) if want_x else None
        loss = torch.empty(1, dtype=torch.float32, device=x.device)
        _check(self.lib.orkan_mlp_gradients(self.h, _ptr(x), _ptr(t), x.shape[0], _ptr(loss), _ptr(g),
                                            None if gx is None else _ptr(gx), _stream()), "gradients")
        return float(loss.item()), g, gx

    def train(self, x, t, epochs, batch=1024, lr=1e-3, seed=0) -> float:
        import torch
        loss = torch.empty(1, dtype=torch.float32, device=x.device)
        _check(self.lib.orkan_mlp_train(self.h, _ptr(x), _ptr(t), x.shape[0], epochs, batch, lr, seed, _ptr(loss),
                                        _stream()), "train")
        return float(loss.item())

    def ascend(self, x, steps=200, lr=0.02, lo=-1.0, hi=1.0):
        """Adam ascent of the network's output over its inputs (in place); returns f(x)."""
        import torch
        y = torch.empty(x.shape[0], dtype=torch.float32, device=x.device)
        _check(self.lib.orkan_mlp_ascend(self.h, _ptr(x), x.shape[0], steps, lr, lo, hi, _ptr(y), _stream()),
               "ascend")
        return y

    def close(self):
        if self.h:
            self.lib.orkan_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------------------
# angle encoding: gamma in [0, pi], beta in [0, pi/2]  <->  inputs in [-1, 1]
# ---------------------------------------------------------------------------------------
def encode(gammas, betas):
    g = np.asarray(gammas, dtype=np.float64) / np.pi * 2.0 - 1.0
    b = np.asarray(betas, dtype=np.float64) / (np.pi / 2.0) * 2.0 - 1.0
    return np.concatenate([g, b], axis=1).astype(np.float32)


def decode(x, p):
    x = np.asarray(x, dtype=np.float64)
    return (x[:, :p] + 1.0) / 2.0 * np.pi, (x[:, p:] + 1.0) / 2.0 * (np.pi / 2.0)


class Evaluator:
    """Exact FP64 expectation values of one cost function at many angle sets: a batch of
    `width` instances of the same graph (one shared cost vector) replayed per call."""

    def __init__(self, ork, n, edges, weights, p, width, tune=True, cache_path=None):
        from .batch import QaoaBatch
        self.p, self.width = p, width
        self.batch = QaoaBatch(ork, [n] * width, [edges] * width, None if weights is None else [weights] * width, p)
        if tune:
            rng = np.random.default_rng(0)
            self.batch.tune(rng.uniform(0, np.pi, (width, p)), rng.uniform(0, np.pi / 2, (width, p)), cache_path)
        self.evals = 0

    def __call__(self, gammas, betas):
        gammas, betas = np.asarray(gammas), np.asarray(betas)
        out = np.empty(len(gammas))
        for c0 in range(0, len(gammas), self.width):
            c1 = min(len(gammas), c0 + self.width)
            g = np.zeros((self.width, self.p))
            b = np.zeros((self.width, self.p))
            g[:c1 - c0], b[:c1 - c0] = gammas[c0:c1], betas[c0:c1]
            out[c0:c1] = self.batch.run(g, b)[:c1 - c0]
            self.evals += c1 - c0
        return out

    def close(self):
        self.batch.close()


def depolarizing_kraus(prob):
    """Kraus operators of the 1-qubit depolarizing channel in the p/4 form of the
    reference's channel tests: sqrt(1 - 3p/4) I, sqrt(p/4) X, Y, Z."""
    a, b = np.sqrt(1.0 - 3.0 * prob / 4.0), np.sqrt(prob / 4.0)
    return [a * np.eye(2), b * np.array([[0, 1], [1, 0]]), b * np.array([[0, -1j], [1j, 0]]),
            b * np.array([[1, 0], [0, -1]])]


def rx_matrix(theta):
    c, s = np.cos(theta / 2.0), np.sin(theta / 2.0)
    return np.array([[c, -1j * s], [-1j * s, c]])


class NoisyEvaluator:
    """Exact FP64 <C> of the noisy circuit on a tiled density matrix through the per-call
    API: state_plus, then per layer exp_diag(cost, gamma_k) and, on every qubit, rx(2 beta_k)
    followed by a depolarizing channel -- applied as one channel_1q with the superoperator
    of the Kraus set {K_i Rx} (kraus_to_superop of the library), then mean(cost)."""

    def __init__(self, ork, n, edges, weights, p, prob, kind="tiled"):
        self.ork, self.n, self.p, self.prob, self.kind = ork, n, p, prob, kind
        x = np.arange(1 << n, dtype=np.int64)
        cost = np.zeros(1 << n)
        for e, (u, v) in enumerate(edges):
            cost += (1.0 if weights is None else float(weights[e])) * (((x >> u) ^ (x >> v)) & 1)
        self.cost = cost
        self.kraus = depolarizing_kraus(prob)
        self.evals = 0

    def one(self, g, b):
        ork = self.ork
        st = ork.plus(self.kind, self.n)
        for k in range(self.p):
            ork.exp_diag(st, self.cost, float(g[k]))
            rx = rx_matrix(2.0 * float(b[k]))
            sop = ork.superop([K @ rx for K in self.kraus])
            for q in range(self.n):
                ork.channel_1q(st, sop, q)
        m = ork.mean(st, self.cost)
        ork.free(st)
        self.evals += 1
        return m

    def __call__(self, gammas, betas):
        return np.array([self.one(g, b) for g, b in zip(np.asarray(gammas), np.asarray(betas))])

    def close(self):
        pass


def plain_sweep(evaluate, p, count, rng, chunk, clock):
    """The method without the network: uniformly random angles in batches; returns the
    samples, their exact values and the best-so-far trace [(seconds, best)]."""
    gs, bs, es, trace = [], [], [], []
    best = -np.inf
    for c0 in range(0, count, chunk):
        c = min(chunk, count - c0)
        g = rng.uniform(0, np.pi, (c, p))
        b = rng.uniform(0, np.pi / 2, (c, p))
        e = evaluate(g, b)
        gs.append(g); bs.append(b); es.append(e)
        best = max(best, float(e.max()))
        trace.append((clock(), best))
    return np.concatenate(gs), np.concatenate(bs), np.concatenate(es), trace


def epochs_for(count, batch=1024, steps=4000, minimum=60):
    """Epochs giving about `steps` Adam steps (at least `minimum` epochs)."""
    return max(minimum, int(np.ceil(steps / max(1, count // batch))))


def fit(net, x, t, batch=1024, lr=1e-3, seed=0, chunk_epochs=5, patience=4, max_epochs=None, val_frac=0.1):
    """Train with early stopping: a fixed 10 % of the pairs is held out, the network trains
    in chunks of `chunk_epochs` epochs on the rest, and the parameters with the lowest
    held-out error are kept.  x, t: numpy arrays (t already normalised).  Returns
    (held-out MSE, epochs trained)."""
    import torch
    dev = torch.device("cuda")
    n = len(t)
    idx = np.random.default_rng(seed).permutation(n)
    nv = max(1, int(n * val_frac))
    tr, va = idx[nv:], idx[:nv]
    batch = min(batch, len(tr))
    xs = torch.from_numpy(np.ascontiguousarray(x[tr])).to(dev)
    ts = torch.from_numpy(np.ascontiguousarray(t[tr]).astype(np.float32)).to(dev)
    xv = torch.from_numpy(np.ascontiguousarray(x[va])).to(dev)
    tv = t[va].astype(np.float64)
    max_epochs = max_epochs or epochs_for(len(tr), batch)
    best, best_p, bad, done = np.inf, net.get_params(), 0, 0
    while done < max_epochs and bad < patience:
        net.train(xs, ts, epochs=chunk_epochs, batch=batch, lr=lr, seed=seed + done)
        done += chunk_epochs
        mse = float(np.mean((net.forward(xv).cpu().numpy().astype(np.float64) - tv) ** 2))
        if mse < best:
            best, best_p, bad = mse, net.get_params(), 0
        else:
            bad += 1
    net.set_params(best_p)
    return best, done


def surrogate_search(ork, evaluate, p, g, b, e, target, clock, rng, hidden=256, batch=1024, rounds=8,
                     proposals=1024, local=4096, radius=0.25, screen=32, seed=1, use_network=True, log=None):
    """Surrogate-guided trust-region search from exactly scored pairs (angles g, b -> e).

    Every round fits the network (early stopping on a held-out 10 %) to the `local` pairs
    nearest to the best point so far -- the landscape is smooth at that scale even where it
    is not over the whole angle box -- draws `screen` x `proposals` candidates uniformly in
    the box of half width `radius` (input units) around that point, keeps the `proposals`
    the network ranks highest, and re-scores them exactly in FP64.  The radius grows after
    a round that improved the best value and shrinks after one that did not.  With
    use_network=False the first `proposals` candidates are scored as drawn (the same search
    without the network).  Stops when the best exact value reaches `target`.
    Returns (best exact value, trace [(seconds, best)], stats)."""
    import torch
    dev = torch.device("cuda")
    all_x = encode(g, b)
    all_e = np.asarray(e, dtype=np.float64)
    net = Mlp(ork, n_in=2 * p, hidden=hidden, max_batch=batch, seed=seed) if use_network else None
    stats = {"train_samples": len(all_e), "train_seconds": 0.0, "validation_r2": [], "epochs": [],
             "radius": [], "proposal_abs_err": []}
    best_i = int(np.argmax(all_e))
    best = float(all_e[best_i])
    trace = [(clock(), best)]
    rad = radius
    for r in range(rounds):
        center = all_x[best_i]
        d = np.max(np.abs(all_x - center), axis=1)
        near = np.argsort(d)[:local]
        lo, hi = np.maximum(center - rad, -1.0), np.minimum(center + rad, 1.0)
        cand = rng.uniform(lo, hi, (screen * proposals, 2 * p)).astype(np.float32)
        stats["radius"].append(rad)
        if net is not None:
            t0 = clock()
            ee = all_e[near]
            mu, sd = float(ee.mean()), float(ee.std()) or 1.0
            val_mse, ep = fit(net, all_x[near], (ee - mu) / sd, batch=min(batch, len(near)), seed=seed + r)
            stats["train_seconds"] += clock() - t0
            stats["validation_r2"].append(1.0 - val_mse)
            stats["epochs"].append(ep)
            y = net.forward(torch.from_numpy(cand).to(dev)).cpu().numpy().astype(np.float64)
            top = np.argsort(-y)[:proposals]
            xq, pred = cand[top], y[top] * sd + mu
        else:
            xq, pred = cand[:proposals], None
        gq, bq = decode(xq, p)
        eq = evaluate(gq, bq)
        if pred is not None:
            stats["proposal_abs_err"].append(float(np.mean(np.abs(pred - eq))))
        improved = float(eq.max()) > best
        all_x = np.concatenate([all_x, xq])
        all_e = np.concatenate([all_e, eq])
        if improved:
            best_i = int(np.argmax(all_e))
            best = float(all_e[best_i])
        rad = min(1.0, rad * 1.5) if improved else max(0.02, rad * 0.5)
        trace.append((clock(), best))
        if log:
            log(f"round {r}: best exact {best:.6f}, radius {rad:.3f}")
        if best >= target:
            break
    stats["rounds"] = len(trace) - 1
    if net is not None:
        net.close()
    return best, trace, stats


def now():
    import torch
    torch.cuda.synchronize()
    return time.perf_counter()
