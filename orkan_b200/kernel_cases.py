"""One kernel class of the single-gate sweep on a reduced state, for profiling.

    python -m orkan_b200.kernel_cases <case> [--pure-qubits 27] [--mixed-qubits 13] [--reps 3]

Runs the case's gates `reps` times on a seeded state after one warm-up round and prints
the algorithmic bytes of every launch (orkan_b200/traffic.py) in launch order, so an ncu
capture of the same command can be set against them.  Cases (the sweep's kernel classes):

  pure_1q_dense   H on qubits 0, n/2, n-1          pure_1q_phase   T on qubits 0, n/2, n-1
  pure_2q         CX (0, n-1), (n-1, 0), (n/2, n/2+1)
  pure_ccx        CCX (0, n/2, n-1), (n-1, n/2, 0), (0, 1, 2)
  tiled_engine / packed_engine   H on 0, 7, n-1;  tiled_ccx / packed_ccx   CCX as above
  tiled_phase / packed_phase     T on 0, 7, n-1;  tiled_exp_diag / packed_exp_diag
  tiled_channel_2q / packed_channel_2q   random 2-qubit channel on (0, n-1), (5, 6)
  pure_fused      a 48-gate random circuit, fused
  pure_fused_costs   crafted runs (1-48 gates, 1-8 register stages), each queued and flushed
                  as one fused launch, timed with CUDA events (prints ms per launch)
The states are larger than L2 at the default sizes (2 GiB statevector, 0.5 GB density
matrices), so DRAM figures are meaningful, and small enough for a short capture.
"""
from __future__ import annotations

import argparse
import sys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("case")
    ap.add_argument("--pure-qubits", type=int, default=27)
    ap.add_argument("--mixed-qubits", type=int, default=13)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args(argv)
    import numpy as np
    import torch

    import orkan_b200
    from orkan_b200 import traffic as T
    from orkan_b200 import workloads as W

    ork = orkan_b200.load(5)
    ork.set_stream(torch.cuda.current_stream().cuda_stream)
    case = args.case
    kind = case.split("_")[0]
    n = args.pure_qubits if kind == "pure" else args.mixed_qubits
    h = n // 2
    ork.set_gate_fusion(48 if case.startswith("pure_fused") else 0)
    st = ork.state(kind, n)
    W.fill_state_on_device(ork, st, kind, n, seed=1, log_tile=5)
    ops = []                                           # (callable, algorithmic bytes)

    def gate(name, qs, th=None):
        ops.append((lambda: ork.gate(st, name, qs, th), T.gate_bytes(kind, n, name, qs, 5)))

    if case.endswith("1q_dense") or case.endswith("_engine"):
        for q in (0, 7 if kind != "pure" else h, n - 1):
            gate("h", (q,))
    elif case.endswith("_phase"):
        for q in (0, 7 if kind != "pure" else h, n - 1):
            gate("t", (q,))
    elif case == "pure_2q":
        for qs in ((0, n - 1), (n - 1, 0), (h, h + 1)):
            gate("cx", qs)
    elif case.endswith("_ccx"):
        for qs in ((0, h, n - 1), (n - 1, h, 0), (0, 1, 2)):
            gate("ccx", qs)
    elif case.endswith("_exp_diag"):
        diag = W.uniform_obs_torch(n, seed=3)
        ops.append((lambda: ork.exp_diag(st, diag.data_ptr(), 0.41), T.exp_diag_bytes(kind, n, 5)))
    elif case.endswith("_channel_2q"):
        rng = np.random.default_rng(2)
        iso, _ = np.linalg.qr(rng.standard_normal((16, 4)) + 1j * rng.standard_normal((16, 4)))
        sop = ork.superop([iso[4 * i:4 * i + 4, :] for i in range(4)])
        for qs in ((0, n - 1), (5, 6)):
            ops.append((lambda qs=qs: ork.channel_2q(st, sop, *qs), T.gate_bytes(kind, n, "h", (0,), 5)))
    elif case == "pure_fused":
        circ = W.random_circuit(n, 48, seed=5)
        alg = sum(T.gate_bytes(kind, n, g, qs, 5) for g, qs, _ in circ)

        def run():
            for g, qs, th in circ:
                ork.gate(st, g, qs, th)
            ork.flush()
        ops.append((run, alg))
    elif case == "pure_fused_costs":
        runs = [("1 H on qubit 0", [("h", (0,), None)]),
                ("8 H on qubits 0-2", [("h", (q % 3,), None) for q in range(8)]),
                ("24 H on qubits 0-2", [("h", (q % 3,), None) for q in range(24)]),
                ("48 H on qubits 0-2", [("h", (q % 3,), None) for q in range(48)]),
                ("24 Rx on qubits 0-2", [("rx", (q % 3,), 0.3) for q in range(24)]),
                ("24 T on qubits 0-2", [("t", (q % 3,), None) for q in range(24)]),
                ("24 CX within qubits 0-2", [("cx", (q % 3, (q + 1) % 3), None) for q in range(24)]),
                (f"24 CX, control qubit {n - 1}, targets 0-2", [("cx", (n - 1, q % 3), None) for q in range(24)]),
                ("6 H on qubits 0-5", [("h", (q,), None) for q in range(6)]),
                ("9 H on qubits 0-8", [("h", (q,), None) for q in range(9)]),
                ("11 H on qubits 0-10", [("h", (q,), None) for q in range(11)]),
                ("24 H cycling over qubits 0-8", [("h", (q % 9,), None) for q in range(24)])]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for label, circ in runs:
            def run(circ=circ):
                for g, qs, th in circ:
                    ork.gate(st, g, qs, th)
                ork.flush()
            for _ in range(2):
                run()
            torch.cuda.synchronize()
            e0.record()
            for _ in range(10 * args.reps):
                run()
            e1.record()
            torch.cuda.synchronize()
            print(f"{label}: {e0.elapsed_time(e1) / (10 * args.reps):.3f} ms per launch")
        ork.free(st)
        return 0
    else:
        print(f"unknown case {case}", file=sys.stderr)
        return 2
    for f, _ in ops:                                  # warm-up round
        f()
    torch.cuda.synchronize()
    for _ in range(args.reps):
        for f, b in ops:
            f()
            print(b)
    torch.cuda.synchronize()
    ork.free(st)
    return 0


if __name__ == "__main__":
    sys.exit(main())
