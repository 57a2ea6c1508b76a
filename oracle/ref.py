"""ctypes access to the reference Orkan library compiled from its own sources -- TEST
INFRASTRUCTURE ONLY (a checker; never the measured product).

oracle/Makefile builds oracle/_ref/liborkan_ref_t5.so (LOG_TILE_DIM=5) and
liborkan_ref_t3.so (LOG_TILE_DIM=3) from the reference's src/ tree.  State data of the
reference lives in host memory; state_init takes ownership of a malloc'd buffer
(reference src/state/state.c:60-99), so buffers handed to it come from libc malloc.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_LIBC = C.CDLL("libc.so.6")
_LIBC.malloc.restype = C.c_void_p
_LIBC.malloc.argtypes = [C.c_size_t]

KIND = {"pure": 0, "packed": 1, "tiled": 2}


class StateT(C.Structure):
    _fields_ = [("type", C.c_int), ("data", C.c_void_p), ("qubits", C.c_ubyte)]


class Cplx(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class KrausT(C.Structure):
    _fields_ = [("n_qubits", C.c_ubyte), ("n_terms", C.c_uint64), ("data", C.c_void_p)]


class SuperopT(C.Structure):
    _fields_ = [("n_qubits", C.c_ubyte), ("data", C.c_void_p)]


def ref_path(log_tile: int = 5) -> str:
    return os.path.join(REF_DIR, f"liborkan_ref_t{log_tile}.so")


def available(log_tile: int = 5) -> bool:
    return os.path.exists(ref_path(log_tile))


class RefLib:
    """The reference library; methods mirror the public C API on numpy arrays."""

    def __init__(self, log_tile: int = 5, threads: int | None = None):
        if threads is not None:
            os.environ["OMP_NUM_THREADS"] = str(threads)
        self.log_tile = log_tile
        self.lib = C.CDLL(ref_path(log_tile))
        L = self.lib
        P = C.POINTER(StateT)
        for g in ("x", "y", "z", "h", "s", "sdg", "t", "tdg", "hy"):
            getattr(L, g).argtypes = [P, C.c_ubyte]
        for g in ("rx", "ry", "rz", "p"):
            getattr(L, g).argtypes = [P, C.c_ubyte, C.c_double]
        for g in ("cx", "cy", "cz", "swap_gate"):
            getattr(L, g).argtypes = [P, C.c_ubyte, C.c_ubyte]
        L.ccx.argtypes = [P, C.c_ubyte, C.c_ubyte, C.c_ubyte]
        L.state_init.argtypes = [P, C.c_ubyte, C.POINTER(C.c_void_p)]
        L.state_free.argtypes = [P]
        L.state_plus.argtypes = [P, C.c_ubyte]
        L.state_len.argtypes = [P]
        L.state_len.restype = C.c_uint64
        L.mean.argtypes = [P, C.c_void_p]
        L.mean.restype = C.c_double
        L.matel_diag.argtypes = [P, P, C.c_void_p]
        L.matel_diag.restype = Cplx
        L.exp_diag.argtypes = [P, C.c_void_p, C.c_double]
        L.kraus_to_superop.argtypes = [C.POINTER(KrausT)]
        L.kraus_to_superop.restype = SuperopT
        L.channel_1q.argtypes = [P, C.POINTER(SuperopT), C.c_ubyte]
        L.single_from_mat.argtypes = [P, C.c_ubyte, C.c_void_p]
        L.two_from_mat.argtypes = [P, C.c_ubyte, C.c_ubyte, C.c_void_p]
        L.state_get.argtypes = [P, C.c_uint64, C.c_uint64]
        L.state_get.restype = Cplx
        _LIBC.free.argtypes = [C.c_void_p]

    # ---- states ------------------------------------------------------------------
    def state(self, kind: str, n: int, storage: np.ndarray | None = None) -> StateT:
        s = StateT(KIND[kind], None, 0)
        if storage is None:
            self.lib.state_init(C.byref(s), n, None)
            return s
        arr = np.ascontiguousarray(storage, dtype=np.complex128)
        buf = _LIBC.malloc(arr.nbytes)
        C.memmove(buf, arr.ctypes.data, arr.nbytes)
        p = C.c_void_p(buf)
        self.lib.state_init(C.byref(s), n, C.byref(p))
        return s

    def plus(self, kind: str, n: int) -> StateT:
        s = StateT(KIND[kind], None, 0)
        self.lib.state_plus(C.byref(s), n)
        return s

    def storage(self, s: StateT) -> np.ndarray:
        n = int(self.lib.state_len(C.byref(s)))
        raw = (C.c_double * (2 * n)).from_address(s.data)
        return np.frombuffer(raw, dtype=np.complex128, count=n).copy()

    def free(self, s: StateT) -> None:
        self.lib.state_free(C.byref(s))

    # ---- operations --------------------------------------------------------------
    def gate(self, s: StateT, name: str, qubits, theta: float | None = None) -> None:
        fn = getattr(self.lib, "swap_gate" if name == "swap" else name)
        args = [C.byref(s)] + [int(q) for q in qubits]
        if theta is not None:
            args.append(float(theta))
        fn(*args)

    def mean(self, s: StateT, obs: np.ndarray) -> float:
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        return float(self.lib.mean(C.byref(s), obs.ctypes.data))

    def matel_diag(self, bra: StateT, ket: StateT, obs: np.ndarray) -> complex:
        obs = np.ascontiguousarray(obs, dtype=np.float64)
        r = self.lib.matel_diag(C.byref(bra), C.byref(ket), obs.ctypes.data)
        return complex(r.re, r.im)

    def exp_diag(self, s: StateT, diag: np.ndarray, t: float) -> None:
        diag = np.ascontiguousarray(diag, dtype=np.float64)
        self.lib.exp_diag(C.byref(s), diag.ctypes.data, float(t))

    def superop(self, kraus) -> np.ndarray:
        ks = np.ascontiguousarray(np.stack([np.asarray(k, dtype=np.complex128) for k in kraus]))
        kt = KrausT(1, len(kraus), ks.ctypes.data)
        so = self.lib.kraus_to_superop(C.byref(kt))
        raw = (C.c_double * 32).from_address(so.data)
        out = np.frombuffer(raw, dtype=np.complex128, count=16).copy().reshape(4, 4)
        _LIBC.free(C.c_void_p(so.data))
        return out

    def channel_1q(self, s: StateT, sop: np.ndarray, q: int) -> None:
        arr = np.ascontiguousarray(sop.reshape(-1), dtype=np.complex128)
        so = SuperopT(1, arr.ctypes.data)
        self.lib.channel_1q(C.byref(s), C.byref(so), int(q))

    def single_from_mat(self, s: StateT, q: int, mat_colmajor: np.ndarray) -> None:
        arr = np.ascontiguousarray(mat_colmajor, dtype=np.complex128)
        self.lib.single_from_mat(C.byref(s), int(q), arr.ctypes.data)

    def two_from_mat(self, s: StateT, q1: int, q2: int, mat_colmajor: np.ndarray) -> None:
        arr = np.ascontiguousarray(mat_colmajor, dtype=np.complex128)
        self.lib.two_from_mat(C.byref(s), int(q1), int(q2), arr.ctypes.data)
