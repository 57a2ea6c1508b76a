"""Python side of the CPU kernel emulator (tests/emu/libkemu.so) -- test infrastructure.

Maps each gate to the kernel-layer operation the host C layer uses for it
(orkan_b200/csrc/host/gate.c), runs the emulated launch and returns the new storage with
per-element read/write counts and the number of out-of-range accesses.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "emu", "libkemu.so")
R2 = 0.70710678118654752440
LAYOUT = {"pure": 0, "packed": 1, "tiled": 2}


def build() -> str:
    src = os.path.join(HERE, "emu", "emu.cpp")
    deps = [src] + [os.path.join(HERE, "..", "orkan_b200", "csrc", "cuda", f)
                    for f in ("common.cuh", "dm_engine.cuh", "dm_phase.cuh", "pure.cuh", "pure_fused.cuh", "qaoa.cuh")]
    deps.append(os.path.join(HERE, "..", "include", "orkan_cu.h"))
    if not os.path.exists(LIB) or any(os.path.getmtime(d) > os.path.getmtime(LIB) for d in deps):
        import subprocess
        cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
        subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-I" + os.path.join(cuda, "include"),
                        src, "-o", LIB], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
    return _lib


def _u32(n):
    return np.zeros(n, dtype=np.uint32)


def _arr(x, dt):
    return np.ascontiguousarray(x, dtype=dt)


class Result:
    def __init__(self, out, reads, writes, oob):
        self.out, self.reads, self.writes, self.oob = out, reads, writes, oob


def _run(fn, data, make_args):
    out = np.array(data, dtype=np.complex128, copy=True)
    reads, writes = _u32(out.size), _u32(out.size)
    oob = C.c_uint64(0)
    rc = fn(*make_args(out, reads, writes, oob))
    if rc != 0:
        raise RuntimeError("emulated launch rejected its parameters")
    return Result(out, reads, writes, oob.value)


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


# kernel-layer ops -------------------------------------------------------------------
def dm_unitary(layout, lt, data, n, qubits, u):
    q = _arr(qubits, np.uint32)
    uu = _arr(np.asarray(u, dtype=np.complex128).reshape(-1), np.complex128)
    f = lib().emu_dm_unitary
    return _run(f, data, lambda o, r, w, b: (LAYOUT[layout], lt, _ptr(o), C.c_uint64(o.size), n, len(q), _ptr(q),
                                             _ptr(uu), _ptr(r), _ptr(w), C.byref(b)))


def dm_monomial(layout, lt, data, n, qubits, src, phase):
    q = _arr(qubits, np.uint32)
    s = _arr(src, np.uint32)
    ph = _arr(phase, np.complex128)
    f = lib().emu_dm_monomial
    return _run(f, data, lambda o, r, w, b: (LAYOUT[layout], lt, _ptr(o), C.c_uint64(o.size), n, len(q), _ptr(q),
                                             _ptr(s), _ptr(ph), _ptr(r), _ptr(w), C.byref(b)))


def dm_phase(layout, lt, data, n, qubits, phase):
    q = _arr(qubits, np.uint32)
    ph = _arr(phase, np.complex128)
    f = lib().emu_dm_phase
    return _run(f, data, lambda o, r, w, b: (LAYOUT[layout], lt, _ptr(o), C.c_uint64(o.size), n, len(q), _ptr(q),
                                             _ptr(ph), _ptr(r), _ptr(w), C.byref(b)))


def dm_superop1(layout, lt, data, n, target, sop):
    s = _arr(np.asarray(sop).reshape(-1), np.complex128)
    f = lib().emu_dm_superop1
    return _run(f, data, lambda o, r, w, b: (LAYOUT[layout], lt, _ptr(o), C.c_uint64(o.size), n, target, _ptr(s),
                                             _ptr(r), _ptr(w), C.byref(b)))


def dm_superop2(layout, lt, data, n, q0, q1, sop):
    s = _arr(np.asarray(sop).reshape(-1), np.complex128)
    f = lib().emu_dm_superop2
    return _run(f, data, lambda o, r, w, b: (LAYOUT[layout], lt, _ptr(o), C.c_uint64(o.size), n, q0, q1, _ptr(s),
                                             _ptr(r), _ptr(w), C.byref(b)))


def dm_exp_diag(layout, lt, data, n, diag, t):
    dg = _arr(diag, np.float64)
    f = lib().emu_dm_exp_diag
    f.argtypes = None
    return _run(f, data, lambda o, r, w, b: (LAYOUT[layout], lt, _ptr(o), C.c_uint64(o.size), n, _ptr(dg),
                                             C.c_double(t), _ptr(r), _ptr(w), C.byref(b)))


PURE_OP1 = {g: i for i, g in enumerate(("x", "y", "z", "h", "s", "sdg", "t", "tdg", "hy", "rx", "ry", "rz", "p"))}
PURE_OP2 = {"cx": 0, "cy": 1, "cz": 2, "swap": 3}


def pure_gate(data, n, name, qubits, theta=None):
    lb = lib()
    if name in PURE_OP1:
        c = s = 0.0
        if name in ("rx", "ry", "rz"):
            c, s = np.cos(theta / 2.0), np.sin(theta / 2.0)
        elif name == "p":
            c, s = np.cos(theta), np.sin(theta)
        return _run(lb.emu_pure_gate1, data, lambda o, r, w, b: (_ptr(o), n, int(qubits[0]), PURE_OP1[name],
                                                                   C.c_double(c), C.c_double(s), _ptr(r), _ptr(w),
                                                                   C.byref(b)))
    if name in PURE_OP2:
        return _run(lb.emu_pure_gate2, data, lambda o, r, w, b: (_ptr(o), n, int(qubits[0]), int(qubits[1]),
                                                                   PURE_OP2[name], _ptr(r), _ptr(w), C.byref(b)))
    return _run(lb.emu_pure_ccx, data, lambda o, r, w, b: (_ptr(o), n, int(qubits[0]), int(qubits[1]),
                                                            int(qubits[2]), _ptr(r), _ptr(w), C.byref(b)))


FUSED_OP = dict(PURE_OP1, cx=16, cy=17, cz=18, swap=19, ccx=20)


class FGate(C.Structure):
    """orkan_fgate_t of include/orkan_cu.h."""
    _fields_ = [("op", C.c_int), ("q", C.c_uint * 3), ("c", C.c_double), ("s", C.c_double)]


def fused_gates(gates):
    """[(name, qubits, theta)] -> an orkan_fgate_t array with the host-computed c, s."""
    arr = (FGate * len(gates))()
    for i, (name, qs, th) in enumerate(gates):
        c = s = 0.0
        if name in ("rx", "ry", "rz"):
            c, s = np.cos(th / 2.0), np.sin(th / 2.0)
        elif name == "p":
            c, s = np.cos(th), np.sin(th)
        q = list(qs) + [0] * (3 - len(qs))
        arr[i] = FGate(FUSED_OP[name], (C.c_uint * 3)(*q), c, s)
    return arr


def pure_fused(data, n, log_chunk, gates, grid_cap=0):
    arr = fused_gates(gates)
    return _run(lib().emu_pure_fused, data, lambda o, r, w, b: (_ptr(o), n, log_chunk, len(gates), arr,
                                                                  grid_cap, _ptr(r), _ptr(w), C.byref(b)))


def fused_stages(n, log_chunk, gates):
    arr = fused_gates(gates)
    return int(lib().emu_fused_stages(n, log_chunk, len(gates), arr))


def fused_need(name, qubits):
    lb = lib()
    lb.emu_fused_need.restype = C.c_ulonglong
    arr = fused_gates([(name, qubits, 0.5)])
    return int(lb.emu_fused_need(arr))


def pure_exp_diag(data, n, diag, t):
    dg = _arr(diag, np.float64)
    return _run(lib().emu_pure_exp_diag, data, lambda o, r, w, b: (_ptr(o), n, _ptr(dg), C.c_double(t), _ptr(r),
                                                                     _ptr(w), C.byref(b)))


def fill(length, value, corner_log_tile=0, corner_dim=0):
    data = np.zeros(length, dtype=np.complex128)
    return _run(lib().emu_fill, data, lambda o, r, w, b: (_ptr(o), C.c_uint64(length), C.c_double(value.real),
                                                           C.c_double(value.imag), corner_log_tile,
                                                           C.c_uint64(corner_dim), _ptr(r), _ptr(w), C.byref(b)))


def dm_gate(layout, lt, data, n, name, qubits, theta=None):
    """The kernel-layer call the host C layer makes for this gate (gate.c)."""
    q = list(qubits)
    if name == "x":
        return dm_monomial(layout, lt, data, n, q, [1, 0], [1, 1])
    if name == "y":
        return dm_monomial(layout, lt, data, n, q, [1, 0], [-1j, 1j])
    if name in ("z", "s", "sdg", "t", "tdg", "p", "rz"):
        ph1 = {"z": -1, "s": 1j, "sdg": -1j, "t": R2 + 1j * R2, "tdg": R2 - 1j * R2}.get(name)
        if ph1 is None:
            ph1 = np.cos(theta) + 1j * np.sin(theta)
        return dm_phase(layout, lt, data, n, q, [1, ph1])
    if name == "h":
        return dm_unitary(layout, lt, data, n, q, [[R2, R2], [R2, -R2]])
    if name == "hy":
        return dm_unitary(layout, lt, data, n, q, [[R2, -R2], [R2, R2]])
    if name in ("rx", "ry"):
        c, s = np.cos(theta / 2.0), np.sin(theta / 2.0)
        u = [[c, -1j * s], [-1j * s, c]] if name == "rx" else [[c, -s], [s, c]]
        return dm_unitary(layout, lt, data, n, q, u)
    if name == "cx":
        return dm_monomial(layout, lt, data, n, q, [0, 1, 3, 2], [1, 1, 1, 1])
    if name == "cy":
        return dm_monomial(layout, lt, data, n, q, [0, 1, 3, 2], [1, 1, -1j, 1j])
    if name == "cz":
        return dm_phase(layout, lt, data, n, q, [1, 1, 1, -1])
    if name == "swap":
        return dm_monomial(layout, lt, data, n, q, [0, 2, 1, 3], [1, 1, 1, 1])
    if name == "ccx":
        return dm_monomial(layout, lt, data, n, q, [0, 1, 2, 3, 4, 5, 7, 6], [1] * 8)
    raise ValueError(name)


def qaoa(n, cost, p, gammas, betas, log_chunk, nthr=64, upto=None, byte_cost=False):
    """Fused QAOA passes 0..upto of one instance; returns (Result over psi, mean or None)."""
    dim = 1 << n
    cd = _arr(cost, np.float64)
    cb = np.zeros(max(16, (dim + 15) // 16 * 16), np.uint8)        # whole 16-byte units, as on the device
    if byte_cost:
        cb[:dim] = np.asarray(cost, dtype=np.uint8)
    g = _arr(gammas, np.float64)
    bt = _arr(betas, np.float64)
    mean = C.c_double(float("nan"))
    up = p if upto is None else upto
    res = _run(lib().emu_qaoa, np.zeros(dim, dtype=np.complex128),
               lambda o, r, w, b: (n, _ptr(cd), _ptr(cb), int(byte_cost), p, _ptr(g), _ptr(bt), log_chunk, nthr, up,
                                   _ptr(o), C.byref(mean), _ptr(r), _ptr(w), C.byref(b)))
    return res, (None if np.isnan(mean.value) else mean.value)
