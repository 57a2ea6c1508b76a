#!/usr/bin/env python
"""Single-gate throughput sweep of the Orkan state-update path on B200.

Workload (one "step"): the sweep of orkan_b200/workloads.sweep() -- every 1-qubit gate on
every target, CX/CY/CZ/SWAP on (low, high), (high, low) and adjacent pairs, CCX on spread
and adjacent triples -- applied to a 30-qubit PURE statevector (16 GiB, Gaussian random,
normalised) and to 14-qubit density matrices in the tiled and the packed layout
(Dirichlet(1,1,1,1) mixtures of 4 Gaussian pure states, 2.15 GB each).  Rotation angles
are uniform in [0, 2 pi).  Inputs are larger than the 126 MB L2, so no flush is needed.

Metric: GB/s of algorithmic bytes (orkan_b200/traffic.py: 2 x 32 B x sectors that hold an
element the gate may change) over device time.  `value` times the sweep on resident
states with CUDA events; `e2e` repeats it through the public C API from pinned host
buffers (state upload, sweep, mean() of a [-1, 1] observable passed as a host pointer,
result read back), copies inside the timed region: every step copies its states, the next
step's copies overlapping this step's gates (orkan_state_upload_async, two device state
sets), and the observables are staged once through the library's host-array cache.

  python bench.py [--gpus N --steps K --warmup W]            # this library on N GPUs
  python bench.py --impl reference [...]                     # the reference CPU library
Multi-GPU: replicas (each rank runs the whole workload on its GPU; no collective on the
data path); value = all ranks' bytes / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "gate/channel GB/s (single-gate throughput sweep)"
UNIT = "GB/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["orkan", "reference"], default="orkan")
    ap.add_argument("--pure-qubits", type=int, default=30)
    ap.add_argument("--mixed-qubits", type=int, default=14)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="budget of the CPU baseline sample")
    ap.add_argument("--batch-instances", type=int, default=4096, help="instances of the batched QAOA leg (0: skip)")
    ap.add_argument("--batch-check", type=int, default=-1,
                    help="batch instances checked against the per-call path (-1: every instance)")
    ap.add_argument("--surrogate-pairs", type=int, default=65536,
                    help="training pairs of the surrogate leg (65536: the configured size; 0: skip)")
    ap.add_argument("--circuit-gates", type=int, default=200,
                    help="gates of the fused-circuit leg on the PURE statevector (0: skip)")
    ap.add_argument("--channel-qubits", type=int, default=13,
                    help="density-matrix qubits of the Kraus-channel leg (0: skip)")
    ap.add_argument("--noisy-pairs", type=int, default=4096,
                    help="training pairs of the noisy (12 q density-matrix) surrogate leg (0: skip)")
    return ap.parse_args()


def reduce_max(x: float, dist, device) -> float:
    """The maximum of x over all ranks of the process group (x itself without one)."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world: int, steps: int, bytes_per_step: float, max_ms: float) -> float:
    """Whole-job GB/s of N replicas: every rank's bytes over the slowest rank's time."""
    return world * steps * bytes_per_step / (max_ms * 1e-3) / 1e9


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def kernel_class(kind: str, name: str) -> str:
    from orkan_b200 import traffic as T
    if kind == "pure":
        if name in ("cx", "cy", "cz", "swap"):
            return "pure_2q"
        if name == "ccx":
            return "pure_ccx"
        return "pure_1q_dense" if (name in T.DENSE_1Q or name == "rz") else "pure_1q_phase"
    if name in T.PHASE_1Q or name == "cz":
        return f"{kind}_phase"
    return f"{kind}_engine"


def build_plan(npure: int, nmix: int, log_tile: int = 5):
    """[(kind, n, name, qubits, theta, bytes, class)] for one step."""
    from orkan_b200 import traffic as T
    from orkan_b200 import workloads as W
    plan = []
    for kind, n in (("pure", npure), ("tiled", nmix), ("packed", nmix)):
        for name, qs, th in W.sweep(n):
            plan.append((kind, n, name, qs, th, T.gate_bytes(kind, n, name, qs, log_tile), kernel_class(kind, name)))
    return plan


# ---------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.proc:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=10)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return out
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        out["samples"] = len(rows)
        out["sm_mhz"] = sm[len(sm) // 2] if sm else None
        try:
            out["sm_max_mhz"] = float(rows[0][2])
        except ValueError:
            pass
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = set()
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        out["reasons"] = sorted(reasons)
        try:
            out["power_w_max"] = max(float(r[3]) for r in rows)
        except ValueError:
            pass
        return out


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "kernel_classes_dram_27q_13q.md")


def profiled_traffic():
    """ncu DRAM traffic of each kernel class from the committed summary's table: {class:
    (DRAM bytes per captured launch, algorithmic bytes of that launch)}.  Table rows are
    `| <class> (<gates>) | <kernel> | <launches> | <algorithmic MB> | <DRAM MB> | <ratio> |`."""
    out = {}
    try:
        with open(PROFILE_TRAFFIC) as f:
            lines = f.readlines()
    except OSError:
        return out
    for line in lines:
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) != 6 or not cells[0] or cells[0].startswith(("case", "---")):
            continue
        try:
            alg, dram = float(cells[3]) * 1e6, float(cells[4]) * 1e6
        except ValueError:
            continue
        out[cells[0].split()[0]] = (dram, alg)
    return out


# ---------------------------------------------------------------------------------------
# CPU reference (the reference library compiled from its own sources, oracle/_ref)
# ---------------------------------------------------------------------------------------
def reference_lib(threads: int):
    os.environ["OMP_NUM_THREADS"] = str(threads)
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    from oracle import ref
    if not ref.available(5):
        return None
    return ref.RefLib(5)


def reference_states(lib, npure, nmix, seed=1):
    from orkan_b200 import workloads as W
    states = {}
    for kind, n in (("pure", npure), ("tiled", nmix), ("packed", nmix)):
        storage = W.initial_storage(kind, n, seed, log_tile=5)
        states[kind] = lib.state(kind, n, storage)
        del storage
    return states


def time_reference_sample(lib, states, plan, stride, offset):
    """Run every stride-th plan entry (starting at offset); return (bytes, seconds)."""
    nbytes, secs = 0, 0.0
    for i, (kind, n, name, qs, th, b, _) in enumerate(plan):
        if i % stride != offset % stride:
            continue
        t0 = time.perf_counter()
        lib.gate(states[kind], name, qs, th)
        secs += time.perf_counter() - t0
        nbytes += b
    return nbytes, secs


# The reference's CPU sample: every SAMPLE_STRIDE-th gate of the sweep (76 of its 1056 gate
# applications, about 8 s on 16 host cores), the same gates in the cpu_baseline of the GPU
# arm and in every step of the reference arm.
SAMPLE_STRIDE = 14


def sweep_config(npure: int, nmix: int, plan) -> dict:
    """The workload description shared by both arms."""
    return {"workload": f"single-gate throughput sweep: {npure} q PURE statevector + {nmix} q tiled and packed "
                        f"density matrices, {len(plan)} gate applications per step",
            "pure_qubits": npure, "mixed_qubits": nmix, "gates_per_step": len(plan),
            "algorithmic_bytes_per_step": sum(e[5] for e in plan),
            "l2": (f"inputs larger than L2 ({16 * 2 ** npure / 2 ** 30:g} GiB and "
                   f"{16 * (2 ** nmix) * (2 ** nmix + 1) / 2 / 1e9:.3g} GB states vs 126 MB L2); no flush")}


def sample_text(plan, cores, secs=None) -> str:
    nsel = len(plan[::SAMPLE_STRIDE])
    t = f", {secs:.1f} s" if secs is not None else ""
    npure = next(e[1] for e in plan if e[0] == "pure")
    nmix = next(e[1] for e in plan if e[0] != "pure")
    return (f"every {SAMPLE_STRIDE}th gate of the sweep ({nsel} of {len(plan)} gate applications{t}) on the same "
            f"states ({npure} q PURE, {nmix} q tiled, {nmix} q packed), OpenMP threads = {cores}")


def cpu_baseline(plan, npure, nmix, budget_s):
    cores = host_cores()
    lib = reference_lib(cores)
    if lib is None:
        return None
    states = reference_states(lib, npure, nmix)
    lib.gate(states["pure"], "h", (0,))                    # warm the pages
    nbytes, secs = time_reference_sample(lib, states, plan, SAMPLE_STRIDE, 0)
    for s in states.values():
        lib.free(s)
    return {"value": nbytes / secs / 1e9, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": sample_text(plan, cores, secs)}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    plan = build_plan(args.pure_qubits, args.mixed_qubits)
    cores = host_cores()
    lib = reference_lib(cores)
    config = dict(sweep_config(args.pure_qubits, args.mixed_qubits, plan), parallelism="replicas x1")
    if lib is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/liborkan_ref_t5.so not built"}))
        return 0
    states = reference_states(lib, args.pure_qubits, args.mixed_qubits)
    for w in range(args.warmup):
        time_reference_sample(lib, states, plan, SAMPLE_STRIDE, 0)
    tot_b, tot_s = 0, 0.0
    for k in range(args.steps):
        b, s = time_reference_sample(lib, states, plan, SAMPLE_STRIDE, 0)
        tot_b += b
        tot_s += s
    value = tot_b / tot_s / 1e9
    sample = sample_text(plan, cores) + f" per step ({args.steps} steps, {tot_s:.1f} s of gate time)"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded Gaussian states, Dirichlet mixtures, uniform angles)", "config": config,
            "sample": sample,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------------------
# observables on the sweep's states: mean, matel_diag (PURE), exp_diag
# ---------------------------------------------------------------------------------------
def observables_leg(args, ork, states, obs_dev):
    import torch
    from orkan_b200 import traffic as T
    peak, peak_kind = measured_peak()
    out = {"unit": "GB/s", "peak": peak, "peak_source": peak_kind}
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def timed(fn, reps=5):
        fn()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    for kind, st in states.items():
        n = args.pure_qubits if kind == "pure" else args.mixed_qubits
        o = obs_dev[kind].data_ptr()
        res = {}
        ms = timed(lambda: ork.mean(st, o))
        res["mean"] = {"ms": ms, "GB/s": T.mean_bytes(kind, n) / (ms * 1e-3) / 1e9}
        if kind == "pure":
            ket = ork.copy(st)                                  # a distinct ket: both arrays come from HBM
            ms = timed(lambda: ork.matel_diag(st, ket, o))
            ork.free(ket)
            b = 40 * (1 << n)                                   # bra, ket (16 B each) and obs (8 B)
            res["matel_diag"] = {"ms": ms, "GB/s": b / (ms * 1e-3) / 1e9}
        else:
            res["mean"]["note"] = "reads the d diagonal elements only: latency-bound, not a bandwidth figure"
        ms = timed(lambda: ork.exp_diag(st, o, 0.37), reps=3)
        res["exp_diag"] = {"ms": ms, "GB/s": T.exp_diag_bytes(kind, n, 5) / (ms * 1e-3) / 1e9}
        for v in res.values():
            v["frac"] = v["GB/s"] / peak
        out[kind] = res
    return out

# ---------------------------------------------------------------------------------------
# fused-circuit leg: a random circuit on the PURE statevector with gate fusion on and off
# ---------------------------------------------------------------------------------------
def circuit_leg(args, ork, clocks_cls, local):
    """A random circuit of the parity configuration's kind (gates uniform over the 18 calls,
    distinct qubits uniform, angles U[0, 2 pi)) on the 30-qubit statevector, timed through
    the public gate calls with statevector gate fusion on (runs of gates per pass) and off
    (one pass per gate).  Reports gates/s, the passes over the state each way, and the
    algorithmic bytes per gate (one dense pass = 2 x 16 GiB) over the time of the run."""
    import torch
    from orkan_b200 import traffic as T
    from orkan_b200 import workloads as W
    n, ng = args.pure_qubits, args.circuit_gates
    gates = W.random_circuit(n, ng, seed=2024)
    alg = sum(T.gate_bytes("pure", n, g, qs, 5) for g, qs, _ in gates)
    st = ork.state("pure", n)
    W.fill_state_on_device(ork, st, "pure", n, seed=11, log_tile=5)
    peak, peak_kind = measured_peak()
    out = {"metric": "circuit gates/s", "config": {"workload": f"{ng}-gate random circuit (gates uniform over the "
                                                               f"18 calls, distinct qubits uniform, angles U[0, 2 pi)) "
                                                               f"on the {n} q PURE statevector",
                                                   "gates": ng, "algorithmic_bytes": alg}}
    for label, cap in (("fused", 48), ("unfused", 0)):
        ork.set_gate_fusion(cap)
        for _ in range(2):                                   # warm-up
            for g, qs, th in gates:
                ork.gate(st, g, qs, th)
        ork.flush()
        torch.cuda.synchronize()
        steps = max(1, args.steps)
        clk = clocks_cls(local)
        clk.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ork.launches()
        e0.record()
        for _ in range(steps):
            for g, qs, th in gates:
                ork.gate(st, g, qs, th)
            ork.flush()
        e1.record()
        torch.cuda.synchronize()
        clocks = clk.stop()
        launches = (ork.launches() - l0) / steps
        ms = e0.elapsed_time(e1) / steps
        state_bytes = 16 * (1 << n)
        out[label] = {"ms": ms, "gates_per_s": ng / (ms * 1e-3), "launches": launches,
                      "gates_per_launch": ng / launches,
                      "algorithmic_GB/s": alg / (ms * 1e-3) / 1e9,
                      "pass_GB/s": 2 * state_bytes * launches / (ms * 1e-3) / 1e9,
                      "pass_frac_of_peak": 2 * state_bytes * launches / (ms * 1e-3) / 1e9 / peak,
                      "clocks": clocks}
    ork.set_gate_fusion(48)                                  # the library default
    ork.free(st)
    out["speedup"] = out["unfused"]["ms"] / out["fused"]["ms"]
    out["peak_source"] = peak_kind
    return out


# ---------------------------------------------------------------------------------------
# Kraus-channel leg: 13 q tiled and packed density matrices, four channel kinds per qubit
# ---------------------------------------------------------------------------------------
def channels_leg(args, ork, clocks_cls, local):
    import torch
    from orkan_b200 import traffic as T
    from orkan_b200 import workloads as W
    n = args.channel_qubits
    chans = W.channel_set(n, seed=3)
    sops = [(label, ork.superop(kr), q) for label, kr, q in chans]
    import numpy as np
    rng2 = np.random.default_rng(11)
    iso, _ = np.linalg.qr(rng2.standard_normal((16, 4)) + 1j * rng2.standard_normal((16, 4)))
    sop2 = ork.superop([iso[4 * i:4 * i + 4, :] for i in range(4)])
    out = {"metric": "channel GB/s", "unit": "GB/s", "dtype": "f64",
           "config": {"workload": f"{n} q tiled and packed density matrices (Dirichlet(1,1,1,1) mixtures of 4 "
                                  f"Gaussian states): depolarizing p~U[0,0.1], amplitude damping g~U[0,0.2], phase "
                                  f"damping l~U[0,0.2] and a random 4-Kraus CPTP channel on every qubit, as "
                                  f"superoperators; then mean and matel_diag (PURE companion state) of a U[-1,1] "
                                  f"observable", "channels_per_step": len(sops)}}
    peak, peak_kind = measured_peak()
    obs = W.uniform_obs_torch(n, seed=9)
    ones = torch.ones(1 << n, dtype=torch.float64, device="cuda")
    for kind in ("tiled", "packed"):
        st = ork.state(kind, n)
        W.fill_state_on_device(ork, st, kind, n, seed=5, log_tile=5)
        nbytes = sum(T.gate_bytes(kind, n, "h", (q,), 5) for _, _, q in sops)    # dense: every element changes
        for label, sop, q in sops[:8]:                                             # warm-up
            ork.channel_1q(st, sop, q)
        torch.cuda.synchronize()
        clk = clocks_cls(local)
        clk.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(max(1, args.steps)):
            for label, sop, q in sops:
                ork.channel_1q(st, sop, q)
        e1.record()
        torch.cuda.synchronize()
        clocks = clk.stop()
        ms = e0.elapsed_time(e1) / max(1, args.steps)
        m = ork.mean(st, obs.data_ptr())
        out[kind] = {"value": nbytes / (ms * 1e-3) / 1e9, "ms_per_step": ms, "algorithmic_bytes_per_step": nbytes,
                     "frac_of_peak": nbytes / (ms * 1e-3) / 1e9 / peak, "peak_source": peak_kind,
                     "trace_after": ork.mean(st, ones.data_ptr()), "mean": m, "clocks": clocks}
        # 2-qubit channels (channel_2q): the random 4-Kraus CPTP map on (q, q + 5 mod n) for
        # every q; every element changes, 64 FP64 FMA per element
        pairs = [(q, (q + 5) % n) for q in range(n)]
        for q0, q1 in pairs[:3]:
            ork.channel_2q(st, sop2, q0, q1)
        torch.cuda.synchronize()
        e0.record()
        for q0, q1 in pairs:
            ork.channel_2q(st, sop2, q0, q1)
        e1.record()
        torch.cuda.synchronize()
        ms2 = e0.elapsed_time(e1) / len(pairs)
        b2 = T.gate_bytes(kind, n, "h", (0,), 5)
        out[kind]["channel_2q"] = {"value": b2 / (ms2 * 1e-3) / 1e9, "us_per_call": ms2 * 1e3,
                                   "frac_of_peak": b2 / (ms2 * 1e-3) / 1e9 / peak, "calls": len(pairs),
                                   "trace_after": ork.mean(st, ones.data_ptr())}
        ork.free(st)
    # observables: mean on both layouts above; matel_diag is PURE-only in the reference
    pst, ket = ork.state("pure", n), ork.state("pure", n)
    W.fill_state_on_device(ork, pst, "pure", n, seed=6, log_tile=5)
    W.fill_state_on_device(ork, ket, "pure", n, seed=7, log_tile=5)
    out["matel_diag_pure"] = [float(x) for x in (lambda z: (z.real, z.imag))(ork.matel_diag(pst, ket, obs.data_ptr()))]
    ork.free(pst)
    ork.free(ket)
    out["value"] = 0.5 * (out["tiled"]["value"] + out["packed"]["value"])
    return out

# ---------------------------------------------------------------------------------------
# batched QAOA leg: 4096 MaxCut instances of 16..24 qubits, p = 4 (include/orkan_batch.h)
# ---------------------------------------------------------------------------------------
def qaoa_batch_workload(count, p=4, seed=2024):
    import numpy as np
    from orkan_b200.batch import random_regular_graph
    rng = np.random.default_rng(seed)
    ns = rng.integers(16, 25, count)
    edges = [random_regular_graph(int(n), 3, rng) for n in ns]
    g = rng.uniform(0, np.pi, (count, p))
    b = rng.uniform(0, np.pi / 2, (count, p))
    return ns, edges, g, b


def plain_qaoa_mean(lib, n, cost, g, b):
    """The per-call plain path (state_plus, exp_diag, rx on every qubit, mean) through a
    library object with the reference's API: this library (GPU) or the reference (CPU)."""
    st = lib.plus("pure", n)
    for k in range(len(g)):
        lib.exp_diag(st, cost, float(g[k]))
        for q in range(n):
            lib.gate(st, "rx", [q], 2.0 * float(b[k]))
    m = lib.mean(st, cost)
    lib.free(st)
    return m


def batched_cpu_baseline(ns, edges, g, b, budget_s):
    """The reference library's per-call path on the host cores, timed on instances of every
    qubit count of the batch: round robin over the counts, smallest first, one instance of
    each count per round, the first round whole and at most two more while the budget lasts.
    The whole batch's time is the sum over qubit counts of (instances of that count) x
    (measured seconds per instance of that count)."""
    from oracle import restate as R
    cores = host_cores()
    lib = reference_lib(cores)
    if lib is None:
        return None
    by_n = {}
    for i, n in enumerate(ns):
        by_n.setdefault(int(n), []).append(i)
    counts = sorted(by_n)
    t_sum = {n: 0.0 for n in counts}
    done = {n: 0 for n in counts}
    secs, rnd = 0.0, 0
    while True:
        progressed = False
        for n in counts:
            if rnd > 0 and secs > budget_s:
                break
            if rnd >= len(by_n[n]):
                continue
            i = by_n[n][rnd]
            cost = R.maxcut_cost(n, edges[i])
            t0 = time.perf_counter()
            plain_qaoa_mean(lib, n, cost, g[i], b[i])
            dt = time.perf_counter() - t0
            t_sum[n] += dt
            done[n] += 1
            secs += dt
            progressed = True
        rnd += 1
        if secs > budget_s or not progressed or rnd >= 3:
            break
    projected = sum(len(by_n[n]) * t_sum[n] / done[n] for n in counts)
    per_n = ", ".join(f"{n} q: {done[n]}" for n in counts)
    return {"value": len(ns) / projected, "unit": "evals/s", "cores": cores, "kind": "reference",
            "seconds_per_instance": {str(n): t_sum[n] / done[n] for n in counts},
            "sample": f"{sum(done.values())} instances of every qubit count of the batch ({per_n}) through the "
                      f"reference's per-call API ({secs:.1f} s); the {len(ns)}-instance batch's time is the sum "
                      f"over qubit counts of instances x measured seconds per instance, OpenMP threads = {cores}"}


def batched_leg(args, ork, clocks_cls, local, dist=None, rank=0, world=1):
    """The batched QAOA leg.  With N ranks the instances are partitioned by work
    (`shard_instances`), every rank evaluates its share on its GPU and the whole batch's
    means are gathered on every rank (one all-reduce of `count` doubles); the device time
    is the slowest rank's, the e2e time includes the gather."""
    import numpy as np
    import torch
    from orkan_b200.batch import ShardedQaoaBatch
    count, p = args.batch_instances, 4
    ns, edges, g, b = qaoa_batch_workload(count, p)
    sh = ShardedQaoaBatch(ork, ns, edges, None, p, rank=rank, world=world)
    bt = sh.local
    t0 = time.perf_counter()
    sh.tune(g, b, None)
    tune_s = time.perf_counter() - t0
    for _ in range(max(3, args.warmup)):
        sh.run(g, b)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks_cls(local)
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(1, args.steps)
    e0.record()
    for _ in range(steps):
        local_means = sh.run(g, b)          # public API: host angles in, host means out
    e1.record()
    torch.cuda.synchronize()
    ms = reduce_max(e0.elapsed_time(e1) / steps, dist, "cuda")
    clocks = clk.stop()
    # end to end: the same runs plus the gather of the whole batch's means on every rank
    if dist:
        dist.barrier()
    w0 = time.perf_counter()
    for _ in range(steps):
        means = sh.gather(sh.run(g, b), dist, "cuda")
    wall = reduce_max((time.perf_counter() - w0) / steps, dist, "cuda")
    waves, launches = bt.stats() if bt is not None else (0, 0)
    amps = float(sum(2.0 ** int(n) for n in ns))
    per_amp = 16 + (p - 1) * 32 + 16 + (p + 1) * 1          # state traffic of the p + 1 passes, byte costs
    achieved = amps * per_amp / (ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    configs = ({int(n): list(bt.config(int(n))) for n in sorted(set(int(ns[i]) for i in sh.idx))}
               if bt is not None else {})
    line = None
    if rank == 0:
        # instances of this rank's share against the per-call plain path of this library
        # (every instance by default; the gathered vector holds the batch's means)
        nchk = len(sh.idx) if args.batch_check < 0 else min(args.batch_check, len(sh.idx))
        pick = (np.arange(len(sh.idx)) if nchk == len(sh.idx)
                else np.random.default_rng(5).choice(len(sh.idx), nchk, replace=False))
        errs, t_plain, amps_plain = [], 0.0, 0.0
        for j in pick:
            i = int(sh.idx[j])
            cost = bt.cost_vector(int(j))
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            m = plain_qaoa_mean(ork, int(ns[i]), cost, g[i], b[i])
            t_plain += time.perf_counter() - t1
            amps_plain += 2.0 ** int(ns[i])
            errs.append(max(abs(m - means[i]), abs(m - local_means[j])))
        plain_evals = count / (t_plain / amps_plain * amps)
        cpu = (batched_cpu_baseline(ns, edges, g, b, args.cpu_seconds)
               if not args.no_cpu_baseline and world == 1 else None)
        line = {"metric": "batched evals/s", "value": count / (ms * 1e-3), "unit": "evals/s",
                "e2e": {"value": count / wall, "unit": "evals/s", "h2d_bytes_per_step": count * p * (8 + 24),
                        "d2h_bytes_per_step": count * 8},
                "ms_per_batch": ms, "dtype": "f64",
                "config": {"workload": f"{count} QAOA MaxCut instances, qubits uniform 16..24, random 3-regular "
                                       f"graphs (one vertex of degree 2 when n is odd), p = {p}, gamma U[0, pi], "
                                       f"beta U[0, pi/2]",
                           "instances": count, "p": p, "ranks": world, "instances_rank0": len(sh.idx),
                           "waves": waves, "launches_per_run": launches, "tuned": configs,
                           "tune_seconds": tune_s, "per_rank_fields": "waves, launches_per_run and tuned "
                                                                      "describe rank 0's share",
                           "l2": "state vectors 1 MiB..256 MiB per instance, 62 GB per wave: larger than L2"},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak * world, "peak_source": peak_kind,
                             "unit": "GB/s", "frac": achieved / (peak * world),
                             "algorithmic_bytes_per_amplitude": per_amp},
                "checked_vs_plain": {"instances": len(errs), "of": len(sh.idx), "max_abs_err": max(errs),
                                     "tolerance": 1e-12, "passed": bool(max(errs) <= 1e-12),
                                     "seconds": t_plain},
                "plain_per_call_gpu_evals_per_s": plain_evals,
                "speedup_vs_plain_per_call": (count / (ms * 1e-3)) / plain_evals,
                "cpu_baseline": cpu, "clocks": clocks}
    sh.close()
    return line


# ---------------------------------------------------------------------------------------
# surrogate leg: FP32 network trained on the batched simulator's pairs, 24 qubits, p = 6
# ---------------------------------------------------------------------------------------
def surrogate_leg(args, ork, noisy=False):
    """Plain batched sweep vs surrogate-guided search on one cost function: the 24-qubit
    statevector (exact evaluator: the batched simulator), or the noisy variant, a 12-qubit
    tiled density matrix with a depolarizing channel (p = 0.01) on every qubit after each
    mixer layer (exact evaluator: the per-call API)."""
    import numpy as np
    import torch
    from orkan_b200.batch import erdos_renyi_graph
    from orkan_b200.surrogate import (Evaluator, Mlp, NoisyEvaluator, encode, fit, now, plain_sweep,
                                      surrogate_search)
    p = 6
    if noisy:
        n, width, ntrain = 12, 256, args.noisy_pairs
    else:
        n, width, ntrain = 24, 512, args.surrogate_pairs
    rng = np.random.default_rng(77)
    edges = erdos_renyi_graph(n, 0.3, rng)
    w = rng.uniform(0.0, 1.0, len(edges))
    ev = NoisyEvaluator(ork, n, edges, w, p, 0.01) if noisy else Evaluator(ork, n, edges, w, p, width)
    rounds, proposals = 8, min(1024, ntrain // 8)
    t_start = now()
    clock = lambda: now() - t_start
    # the plain batched sweep: uniform random angles, twice the training budget
    g, b, e, trace = plain_sweep(ev, p, 2 * ntrain, np.random.default_rng(1), width, clock)
    t_plain_total = trace[-1][0]
    e_plain = float(e.max())
    k_data = next(k for k in range(len(trace)) if (k + 1) * width >= ntrain)
    t_data = trace[k_data][0]
    # surrogate-guided search: the same sweep's first ntrain pairs, then proposal rounds
    # (its best-so-far trace is the sweep's up to t_data, then its own rounds); the same
    # rounds without the network are the ablation
    def search(use_network):
        s0 = clock()
        best, strace, stats = surrogate_search(ork, ev, p, g[:ntrain], b[:ntrain], e[:ntrain], np.inf, clock,
                                               np.random.default_rng(2), rounds=rounds, proposals=proposals,
                                               use_network=use_network)
        return best, trace[:k_data + 1] + [(t_data + (t - s0), bb) for t, bb in strace], stats, clock() - s0

    best, sur_trace, stats, s_spent = search(True)
    best_abl, abl_trace, _, _ = search(False)

    def time_to(tr, level):
        hit = [t for t, bb in tr if bb >= level]
        return hit[0] if hit else None

    target_plain = e_plain - 1e-3
    target_best = max(e_plain, best) - 1e-3
    # surrogate error on held-out pairs (the sweep's second half), network trained as above
    net = Mlp(ork, 2 * p, 256, 1024, seed=1)
    mu, sd = float(e[:ntrain].mean()), float(e[:ntrain].std())
    fit(net, encode(g[:ntrain], b[:ntrain]), (e[:ntrain] - mu) / sd, seed=1)
    xh = torch.from_numpy(encode(g[ntrain:], b[ntrain:])).cuda()
    pred = net.forward(xh).cpu().numpy().astype(np.float64) * sd + mu
    err = pred - e[ntrain:]
    net.close()
    ev.close()
    if noisy:
        workload = (f"noisy variant: {n}-qubit tiled density matrix, weighted MaxCut (Erdos-Renyi p = 0.3, "
                    f"{len(edges)} edges, weights U[0, 1]), p = {p}, depolarizing p = 0.01 on every qubit after "
                    f"each mixer layer; FP32 MLP 12-256-256-1 GELU")
    else:
        workload = (f"{n}-qubit weighted MaxCut (Erdos-Renyi p = 0.3, {len(edges)} edges, weights U[0, 1]), "
                    f"p = {p} layers; FP32 MLP 12-256-256-1 GELU, Adam, batch 1024")
    return {"metric": "surrogate vs plain time-to-|dE|<=1e-3",
            "config": {"workload": workload, "training_pairs": ntrain, "plain_sweep_evals": 2 * ntrain,
                       "proposals_per_round": proposals, "rounds": stats["rounds"]},
            "plain_best": e_plain, "surrogate_best": best, "no_network_best": best_abl,
            "target_plain_best": {"level": target_plain, "plain_seconds": time_to(trace, target_plain),
                                  "surrogate_seconds": time_to(sur_trace, target_plain),
                                  "no_network_seconds": time_to(abl_trace, target_plain)},
            "target_overall_best": {"level": target_best, "plain_seconds": time_to(trace, target_best),
                                    "surrogate_seconds": time_to(sur_trace, target_best),
                                    "no_network_seconds": time_to(abl_trace, target_best),
                                    "plain_budget_seconds": t_plain_total},
            "surrogate_seconds": {"data": t_data, "train": stats["train_seconds"], "search": s_spent},
            "exact_evals": {"plain": int(len(e)), "surrogate": int(ntrain + proposals * stats["rounds"])},
            "local_validation_r2_per_round": stats["validation_r2"], "radius_per_round": stats["radius"],
            "proposal_abs_err_per_round": stats["proposal_abs_err"],
            "heldout": {"pairs": int(len(err)), "mae": float(np.mean(np.abs(err))),
                        "rmse": float(np.sqrt(np.mean(err ** 2))),
                        "r2": float(1.0 - np.mean(err ** 2) / np.var(e[ntrain:]))},
            "exact_evals_per_s": len(e) / t_plain_total}

# ---------------------------------------------------------------------------------------
# this library on the GPU
# ---------------------------------------------------------------------------------------
def run_gpu(args):
    import numpy as np
    import torch

    import orkan_b200
    from orkan_b200 import workloads as W

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return reduce_max(x, dist, "cuda")

    ork = orkan_b200.load(5)
    ork.set_stream(torch.cuda.current_stream().cuda_stream)
    # the sweep measures one-gate kernels: statevector gate fusion stays off for it (the
    # circuit leg below measures fused runs)
    ork.set_gate_fusion(0)
    plan = build_plan(args.pure_qubits, args.mixed_qubits)
    step_bytes = sum(e[5] for e in plan)

    # states (generated on the device, seeded) and observables
    states, host_in, obs_dev, obs_host, nbytes_state = {}, {}, {}, {}, {}
    pinned = True
    for kind, n in (("pure", args.pure_qubits), ("tiled", args.mixed_qubits), ("packed", args.mixed_qubits)):
        st = ork.state(kind, n)
        W.fill_state_on_device(ork, st, kind, n, seed=1 + rank, log_tile=5)
        states[kind] = st
        obs = W.uniform_obs_torch(n, seed=7)
        obs_dev[kind] = obs
        nbytes_state[kind] = int(ork.lib.state_len(orkan_b200.C.byref(st))) * 16
        if not args.no_e2e:
            try:
                h = torch.empty(nbytes_state[kind] // 16, dtype=torch.complex128, pin_memory=pinned)
                o = torch.empty(1 << n, dtype=torch.float64, pin_memory=pinned)
            except RuntimeError:
                pinned = False
                h = torch.empty(nbytes_state[kind] // 16, dtype=torch.complex128)
                o = torch.empty(1 << n, dtype=torch.float64)
            h.copy_(W.state_view(ork, st))
            o.copy_(obs)
            host_in[kind], obs_host[kind] = h, o
    torch.cuda.synchronize()

    def sweep(record=None, sts=None, only=None):
        sts = states if sts is None else sts
        for i, (kind, n, name, qs, th, b, cls) in enumerate(plan):
            if only is not None and kind != only:
                continue
            ork.gate(sts[kind], name, qs, th)
            if record is not None:
                record[i].record()

    for _ in range(args.warmup):
        sweep()
    torch.cuda.synchronize()

    # ---- device-timed region ----
    ev = [[torch.cuda.Event(enable_timing=True) for _ in plan] for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    launches0 = ork.launches()
    start.record()
    for k in range(args.steps):
        sweep(ev[k])
    end.record()
    torch.cuda.synchronize()
    launches = ork.launches() - launches0
    barrier()
    clk = clocks.stop()
    total_ms = start.elapsed_time(end)
    per_class_ms, per_class_bytes, per_class_n = {}, {}, {}
    for k in range(args.steps):
        prev = start if k == 0 else ev[k - 1][-1]
        for i, e in enumerate(plan):
            dt = prev.elapsed_time(ev[k][i])
            prev = ev[k][i]
            cls = e[6]
            per_class_ms[cls] = per_class_ms.get(cls, 0.0) + dt
            per_class_bytes[cls] = per_class_bytes.get(cls, 0) + e[5]
            per_class_n[cls] = per_class_n.get(cls, 0) + 1
    max_ms = max_over_ranks(total_ms)
    value = replica_value(world, args.steps, step_bytes, max_ms)

    # ---- end to end through the public API with host buffers ----
    # Every step copies its three states from pinned host memory (orkan_state_upload_async)
    # and reads back three means.  Two sets of device states: step k's gates run on set
    # k % 2 while step k + 1's states are copied into the other set on a copy stream (the
    # copy starts after the library's earlier work on that set); the library stream waits
    # for each state's copy before that state's gates.  The density matrices go first (their
    # copies are short, and their gates then run while the statevector's copy is in flight
    # in the first step).  The observables are host arrays passed to mean at every step; the
    # library's host-array cache (orkan_set_host_array_cache) stages each once, so the first
    # step copies them and later steps reuse the device copies.
    e2e = None
    if not args.no_e2e:
        kinds = [(kind, n) for kind, n in (("tiled", args.mixed_qubits), ("packed", args.mixed_qubits),
                                           ("pure", args.pure_qubits))]
        sets = [states, {kind: ork.state(kind, n) for kind, n in kinds}]
        obs_bytes = sum(8 * (1 << n) for _, n in kinds)
        ork.lib.orkan_set_host_array_cache.argtypes = [orkan_b200.C.c_size_t]
        ork.lib.orkan_set_host_array_cache(obs_bytes)
        copy_stream = torch.cuda.Stream()
        lib_stream = torch.cuda.current_stream()

        def enqueue_upload(j):
            done = {}
            for kind, _ in kinds:
                ork.upload_async(sets[j % 2][kind], host_in[kind].data_ptr(), copy_stream.cuda_stream)
                done[kind] = copy_stream.record_event()
            return done

        def e2e_steps(nsteps, results):
            up = enqueue_upload(0)
            for k in range(nsteps):
                nxt = enqueue_upload(k + 1) if k + 1 < nsteps else None
                for kind, _ in kinds:
                    lib_stream.wait_event(up[kind])        # this state of step k is on the device
                    sweep(sts=sets[k % 2], only=kind)
                for kind, _ in kinds:
                    results.append((kind, ork.mean(sets[k % 2][kind], obs_host[kind].data_ptr())))
                up = nxt

        e2e_steps(1, [])                               # untimed: the same code path once
        ork.lib.orkan_host_arrays_changed()            # the timed steps stage the observables again
        barrier()
        torch.cuda.synchronize()
        e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        results = []
        e_start.record()
        e2e_steps(args.steps, results)
        e_end.record()
        torch.cuda.synchronize()
        barrier()
        e_ms = max_over_ranks(e_start.elapsed_time(e_end))
        ork.lib.orkan_set_host_array_cache(0)
        for kind, _ in kinds:
            ork.free(sets[1][kind])
        state_bytes = sum(nbytes_state.values())
        e2e = {"value": world * args.steps * step_bytes / (e_ms * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": state_bytes + obs_bytes // max(1, args.steps),
               "d2h_bytes_per_step": 8 * len(states), "ms_per_step": e_ms / args.steps,
               "pinned_host_buffers": pinned, "state_bytes_copied_per_step": state_bytes,
               "observable_bytes_copied_once": obs_bytes,
               "overlap": "step k+1's state copies run on a copy stream under step k's gates (two device "
                          "state sets); in the first step the density matrices' gates run during the "
                          "statevector's copy",
               "means": {kind: float(x) for kind, x in results[-3:]}}

    # ---- roofline of the dominant kernel ----
    dom = max(per_class_ms, key=per_class_ms.get)
    peak, peak_kind = measured_peak()
    launches_dom = per_class_n[dom]
    avg_ms = per_class_ms[dom] / launches_dom
    avg_bytes = per_class_bytes[dom] / launches_dom
    achieved = avg_bytes / (avg_ms * 1e-3) / 1e9
    prof = profiled_traffic()
    traffic = prof[dom][0] / prof[dom][1] * avg_bytes if dom in prof else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_source": peak_kind,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "algorithmic_bytes_per_launch": avg_bytes, "avg_launch_ms": avg_ms, "launches": launches_dom}
    classes = {c: {"launches": per_class_n[c], "ms": per_class_ms[c], "share": per_class_ms[c] / sum(per_class_ms.values()),
                   "GB/s": per_class_bytes[c] / (per_class_ms[c] * 1e-3) / 1e9} for c in sorted(per_class_ms)}
    # compact per-class table beside the dominant kernel: achieved GB/s, fraction of the
    # measured peak, and ncu DRAM traffic / algorithmic bytes where a capture is committed
    roofline["classes"] = {
        c: {"GB/s": round(v["GB/s"], 1), "frac": round(v["GB/s"] / peak, 3), "share": round(v["share"], 3),
            "traffic_ratio": (round(prof[c][0] / prof[c][1], 3) if c in prof else None)}
        for c, v in classes.items()}
    by_gate = {}
    for k in range(args.steps):
        prev = start if k == 0 else ev[k - 1][-1]
        for i, e in enumerate(plan):
            dt = prev.elapsed_time(ev[k][i])
            prev = ev[k][i]
            key = f"{e[0]}:{e[2]}"
            t = by_gate.setdefault(key, [0.0, 0])
            t[0] += dt
            t[1] += e[5]
    gates = {key: {"ms": v[0], "GB/s": v[1] / (v[0] * 1e-3) / 1e9} for key, v in sorted(by_gate.items())}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # free device memory first is not needed; the CPU baseline runs on host memory
        cpu = cpu_baseline(plan, args.pure_qubits, args.mixed_qubits, args.cpu_seconds)

    observables = observables_leg(args, ork, states, obs_dev) if rank == 0 else None
    for st in states.values():
        ork.free(st)
    ork.set_gate_fusion(48)                  # the library default from here on
    circuit = circuit_leg(args, ork, ClockSampler, local) if rank == 0 and args.circuit_gates > 0 else None
    batched = surrogate = noisy = channels = None
    if rank == 0 and world == 1 and args.channel_qubits > 0:
        channels = channels_leg(args, ork, ClockSampler, local)
    if args.batch_instances > 0:             # every rank: the batch is sharded over the ranks
        batched = batched_leg(args, ork, ClockSampler, local, dist, rank, world)
    if rank == 0 and world == 1 and args.surrogate_pairs > 0:
        surrogate = surrogate_leg(args, ork)
    if rank == 0 and world == 1 and args.noisy_pairs > 0:
        noisy = surrogate_leg(args, ork, noisy=True)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded Gaussian states, Dirichlet mixtures, uniform angles)",
                "config": dict(sweep_config(args.pure_qubits, args.mixed_qubits, plan),
                               parallelism=f"replicas x{world}"),
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
                "gpu_launches": launches, "kernel_classes": classes, "by_gate": gates,
                "observables": observables, "circuit": circuit, "channels": channels, "batched": batched, "surrogate": surrogate, "surrogate_noisy": noisy}
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
