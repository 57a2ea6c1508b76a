"""Generate the golden fixtures of tests/golden from the reference library itself.

Run in a checkout where oracle/_ref has been built from the reference sources
(`make -C oracle`):  python tests/golden/make_golden.py

Every fixture is produced by the reference's own compiled backends (oracle/_ref), on
inputs generated here from fixed seeds, and stored as .npz:

  chain_<layout>_<n>q_t<L>.npz  a chain of every gate on every ordered qubit tuple (rotation
                                angles from a seeded stream), applied one after another to
                                a seeded random input; after each gate the checksum
                                sum_i w_i * storage_i with fixed weights w is recorded, and
                                the final storage is kept.  Tiled chains leave out the two
                                gate patterns where the reference's tiled backend deviates
                                from its documented semantics (SWAP with both qubits at tile
                                level, CCX with all three at tile level).
  channels_<layout>_<n>q_t<L>.npz  the same for 1-qubit channels (depolarizing p/4 form,
                                amplitude damping, phase damping, bit flip) on every qubit.
  circuit_pure_12q.npz, circuit_packed_8q.npz
                                the random 200-gate circuit configuration from |+> (and
                                the 8 q packed density matrix, which also pins the tiled
                                layout), with the final storage and mean of a uniform
                                [-1, 1] observable.
  meas_circ.npz                 mean / matel_diag / exp_diag values on seeded inputs.
"""
import itertools
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref as REF          # noqa: E402
from oracle import restate as R        # noqa: E402
from orkan_b200 import workloads as W  # noqa: E402


def rand_rho(n, seed):
    rng = np.random.default_rng(seed)
    d = 1 << n
    a = rng.standard_normal((d, 3)) + 1j * rng.standard_normal((d, 3))
    rho = a @ a.conj().T
    return rho / np.trace(rho).real


def weights(length, seed=99):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(length) + 1j * rng.standard_normal(length)


def chain_ops(n, kind, lt, seed):
    rng = np.random.default_rng(seed)
    ops = []
    for g in W.ALL_GATES:
        k = W.gate_arity(g)
        if k > n:
            continue
        for qs in itertools.permutations(range(n), k):
            if kind == "tiled" and g in ("swap", "ccx") and min(qs) >= lt:
                continue
            theta = float(rng.uniform(0, 2 * np.pi)) if g in W.GATES_ROT else None
            ops.append((g, qs, theta))
    return ops


def encode_ops(ops):
    names = np.array([o[0] for o in ops])
    qubits = np.array([list(o[1]) + [-1] * (3 - len(o[1])) for o in ops], dtype=np.int64)
    thetas = np.array([np.nan if o[2] is None else o[2] for o in ops])
    return names, qubits, thetas


def make_chain(lib, kind, n, lt):
    start = W.gaussian_pure(n, 5) if kind == "pure" else rand_rho(n, 5)
    storage = R.to_storage(kind, start, lt)
    ops = chain_ops(n, kind, lt, seed=17 + n)
    w = weights(storage.size)
    st = lib.state(kind, n, storage)
    sums = []
    for g, qs, th in ops:
        lib.gate(st, g, qs, th)
        sums.append(np.sum(w * lib.storage(st)))
    final = lib.storage(st)
    lib.free(st)
    names, qubits, thetas = encode_ops(ops)
    np.savez_compressed(os.path.join(HERE, f"chain_{kind}_{n}q_t{lt}.npz"), start=storage, names=names,
                        qubits=qubits, thetas=thetas, checksums=np.array(sums), final=final, weights_seed=99)


def make_channels(lib, kind, n, lt):
    start = R.to_storage(kind, rand_rho(n, 6), lt)
    kraus = [R.depolarizing_kraus(0.07), R.amplitude_damping_kraus(0.15), R.phase_damping_kraus(0.1),
             R.bitflip_kraus(0.3)]
    sops = np.stack([lib.superop(k) for k in kraus])
    w = weights(start.size)
    st = lib.state(kind, n, start)
    sums = []
    for s in sops:
        for q in range(n):
            lib.channel_1q(st, s, q)
            sums.append(np.sum(w * lib.storage(st)))
    final = lib.storage(st)
    lib.free(st)
    np.savez_compressed(os.path.join(HERE, f"channels_{kind}_{n}q_t{lt}.npz"), start=start, superops=sops,
                        checksums=np.array(sums), final=final, weights_seed=99)


def make_circuit(lib, kind, n):
    circ = W.random_circuit(n, 200, seed=2024)
    obs = W.uniform_obs(n, seed=7)
    st = lib.plus(kind, n)
    for g, qs, th in circ:
        lib.gate(st, g, qs, th)
    final = lib.storage(st)
    m = lib.mean(st, obs)
    lib.free(st)
    names, qubits, thetas = encode_ops(circ)
    np.savez_compressed(os.path.join(HERE, f"circuit_{kind}_{n}q.npz"), names=names, qubits=qubits, thetas=thetas,
                        final=final, mean=m, obs_seed=7)


def make_meas(lib):
    out = {}
    for kind in ("pure", "packed", "tiled"):
        for n in (3, 5):
            full = W.gaussian_pure(n, n) if kind == "pure" else rand_rho(n, n)
            rng = np.random.default_rng(100 + n)
            obs = rng.uniform(-1, 1, 1 << n)
            diag = rng.uniform(-4, 4, 1 << n)
            storage = R.to_storage(kind, full, 5)
            st = lib.state(kind, n, storage)
            out[f"{kind}{n}_start"] = storage
            out[f"{kind}{n}_obs"] = obs
            out[f"{kind}{n}_diag"] = diag
            out[f"{kind}{n}_mean"] = lib.mean(st, obs)
            lib.exp_diag(st, diag, 0.83)
            out[f"{kind}{n}_exp_diag"] = lib.storage(st)
            lib.free(st)
    bra, ket = W.gaussian_pure(6, 1), W.gaussian_pure(6, 2)
    obs = np.random.default_rng(3).uniform(-1, 1, 64)
    sb, sk = lib.state("pure", 6, bra), lib.state("pure", 6, ket)
    out["matel_bra"], out["matel_ket"], out["matel_obs"] = bra, ket, obs
    out["matel"] = lib.matel_diag(sb, sk, obs)
    lib.free(sb)
    lib.free(sk)
    np.savez_compressed(os.path.join(HERE, "meas_circ.npz"), **out)


def main():
    lib5, lib3 = REF.RefLib(5), REF.RefLib(3)
    make_chain(lib5, "pure", 5, 5)
    make_chain(lib5, "packed", 4, 5)
    make_chain(lib3, "tiled", 5, 3)
    make_chain(lib5, "tiled", 6, 5)
    make_channels(lib5, "packed", 4, 5)
    make_channels(lib3, "tiled", 5, 3)
    make_circuit(lib5, "pure", 12)
    make_circuit(lib5, "packed", 8)
    make_meas(lib5)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
