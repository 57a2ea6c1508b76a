"""Orkan-B200: Python access to the CUDA library through its C ABI (ctypes).

The product is the shared library orkan_b200/liborkan_b200.so (built by
orkan_b200/build.py): the reference's public C API (state.h, gate.h, channel.h, meas.h,
circ.h) on device-resident state storage, plus the kernel layer of include/orkan_cu.h.
This module is a thin binding used by the tests and the benchmark; every call goes to
the compiled library, and loading fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import library_path

KIND = {"pure": 0, "packed": 1, "tiled": 2}


class StateT(C.Structure):
    """state_t of include/state.h (data is a device pointer)."""
    _fields_ = [("type", C.c_int), ("data", C.c_void_p), ("qubits", C.c_ubyte)]


class Cplx(C.Structure):
    """cplx_t (double _Complex) by value: returned/passed like a struct of two doubles."""
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class KrausT(C.Structure):
    _fields_ = [("n_qubits", C.c_ubyte), ("n_terms", C.c_uint64), ("data", C.c_void_p)]


class SuperopT(C.Structure):
    _fields_ = [("n_qubits", C.c_ubyte), ("data", C.c_void_p)]


QOP = C.CFUNCTYPE(None, C.POINTER(StateT))     # qop_t of include/state.h


class SmChannel(C.Structure):
    """sm_channel_t of include/orkan_sample.h."""
    _fields_ = [("n_ops", C.c_uint), ("ops", C.POINTER(QOP)), ("weights", C.c_void_p)]


class OrkanError(RuntimeError):
    pass


_LOADED: dict[int, "Orkan"] = {}


def load(log_tile: int = 5) -> "Orkan":
    """Load (once per process) the library built for the given LOG_TILE_DIM (5 or 3)."""
    if log_tile not in _LOADED:
        _LOADED[log_tile] = Orkan(log_tile)
    return _LOADED[log_tile]


class Orkan:
    def __init__(self, log_tile: int = 5):
        path = library_path(log_tile)
        if not os.path.exists(path):
            raise OrkanError(f"CUDA library {path} is missing: run orkan_b200/build.py "
                             "(or __graft_entry__.build()) first")
        self.path = path
        self.log_tile = log_tile
        self.lib = C.CDLL(path)
        self._declare()
        if self.lib.orkan_log_tile_dim() != log_tile:
            raise OrkanError("library tile geometry does not match its file name")

    def _declare(self):
        L = self.lib
        P = C.POINTER(StateT)
        vp = C.c_void_p
        for g in ("x", "y", "z", "h", "s", "sdg", "t", "tdg", "hy"):
            getattr(L, g).argtypes = [P, C.c_ubyte]
            getattr(L, g).restype = None
        for g in ("rx", "ry", "rz", "p"):
            getattr(L, g).argtypes = [P, C.c_ubyte, C.c_double]
            getattr(L, g).restype = None
        for g in ("cx", "cy", "cz", "swap_gate"):
            getattr(L, g).argtypes = [P, C.c_ubyte, C.c_ubyte]
            getattr(L, g).restype = None
        L.ccx.argtypes = [P, C.c_ubyte, C.c_ubyte, C.c_ubyte]
        L.state_init.argtypes = [P, C.c_ubyte, C.POINTER(vp)]
        L.state_free.argtypes = [P]
        L.state_plus.argtypes = [P, C.c_ubyte]
        L.state_len.argtypes = [P]
        L.state_len.restype = C.c_uint64
        L.state_cp.argtypes = [P]
        L.state_cp.restype = StateT
        L.state_get.argtypes = [P, C.c_uint64, C.c_uint64]
        L.state_get.restype = Cplx
        L.state_set.argtypes = [P, C.c_uint64, C.c_uint64, Cplx]
        L.mean.argtypes = [P, vp]
        L.mean.restype = C.c_double
        L.matel_diag.argtypes = [P, P, vp]
        L.matel_diag.restype = Cplx
        L.exp_diag.argtypes = [P, vp, C.c_double]
        L.kraus_to_superop.argtypes = [C.POINTER(KrausT)]
        L.kraus_to_superop.restype = SuperopT
        L.channel_1q.argtypes = [P, C.POINTER(SuperopT), C.c_ubyte]
        L.channel_2q.argtypes = [P, C.POINTER(SuperopT), C.c_ubyte, C.c_ubyte]
        L.single_from_mat.argtypes = [P, C.c_ubyte, vp]
        L.two_from_mat.argtypes = [P, C.c_ubyte, C.c_ubyte, vp]
        L.orkan_log_tile_dim.restype = C.c_int
        L.orkan_set_stream.argtypes = [vp]
        L.orkan_get_stream.restype = vp
        L.orkan_state_upload.argtypes = [P, vp]
        L.orkan_state_upload.restype = C.c_int
        L.orkan_state_upload_async.argtypes = [P, vp, vp]
        L.orkan_state_upload_async.restype = C.c_int
        L.orkan_state_download.argtypes = [P, vp]
        L.orkan_state_download.restype = C.c_int
        L.orkan_launch_count.restype = C.c_ulonglong
        L.orkan_debug_fail_allocs.argtypes = [C.c_int]
        L.orkan_cu_launch_count.restype = C.c_ulonglong
        L.sample_matrix.argtypes = [P, vp, C.POINTER(SmChannel), C.c_uint, C.c_uint, C.c_size_t, vp]
        L.sample_matrix.restype = None
        L.orkan_flush.restype = None
        L.orkan_set_gate_fusion.argtypes = [C.c_uint]
        L.orkan_set_gate_fusion.restype = None
        L.orkan_get_gate_fusion.restype = C.c_uint

    # ---- states ------------------------------------------------------------------
    def state(self, kind: str, n: int, storage: np.ndarray | None = None) -> StateT:
        """A zeroed device state, or one holding the given storage array."""
        s = StateT(KIND[kind], None, 0)
        self.lib.state_init(C.byref(s), n, None)
        if not s.data:
            raise OrkanError("device allocation failed")
        if storage is not None:
            self.upload(s, storage)
        return s

    def plus(self, kind: str, n: int) -> StateT:
        s = StateT(KIND[kind], None, 0)
        self.lib.state_plus(C.byref(s), n)
        if not s.data:
            raise OrkanError("device allocation failed")
        return s

    def upload(self, s: StateT, storage: np.ndarray) -> None:
        arr = np.ascontiguousarray(storage, dtype=np.complex128)
        if arr.size != self.lib.state_len(C.byref(s)):
            raise OrkanError("storage length does not match the state")
        rc = self.lib.orkan_state_upload(C.byref(s), arr.ctypes.data)
        if rc:
            raise OrkanError(f"upload failed: CUDA error {rc}")

    def upload_async(self, s: StateT, host_ptr: int, stream: int | None = None) -> None:
        """orkan_state_upload_async: the copy of state_len(s) elements from host_ptr is enqueued
        on stream (a cudaStream_t handle; None: the library stream) after the library stream's
        pending work; the caller keeps the host buffer alive and orders later work after it."""
        rc = self.lib.orkan_state_upload_async(C.byref(s), C.c_void_p(host_ptr), C.c_void_p(stream))
        if rc:
            raise OrkanError(f"upload failed: CUDA error {rc}")

    def storage(self, s: StateT) -> np.ndarray:
        out = np.empty(int(self.lib.state_len(C.byref(s))), dtype=np.complex128)
        rc = self.lib.orkan_state_download(C.byref(s), out.ctypes.data)
        if rc:
            raise OrkanError(f"download failed: CUDA error {rc}")
        return out

    def free(self, s: StateT) -> None:
        self.lib.state_free(C.byref(s))

    def copy(self, s: StateT) -> StateT:
        return self.lib.state_cp(C.byref(s))

    def get(self, s: StateT, r: int, c: int = 0) -> complex:
        v = self.lib.state_get(C.byref(s), r, c)
        return complex(v.re, v.im)

    def set(self, s: StateT, r: int, c: int, val: complex) -> None:
        self.lib.state_set(C.byref(s), r, c, Cplx(val.real, val.imag))

    # ---- operations --------------------------------------------------------------
    def gate(self, s: StateT, name: str, qubits, theta: float | None = None) -> None:
        fn = getattr(self.lib, "swap_gate" if name == "swap" else name)
        args = [C.byref(s)] + [int(q) for q in qubits]
        if theta is not None:
            args.append(float(theta))
        fn(*args)

    def mean(self, s: StateT, obs) -> float:
        ptr = obs if isinstance(obs, int) else np.ascontiguousarray(obs, dtype=np.float64).ctypes.data
        return float(self.lib.mean(C.byref(s), ptr))

    def matel_diag(self, bra: StateT, ket: StateT, obs) -> complex:
        ptr = obs if isinstance(obs, int) else np.ascontiguousarray(obs, dtype=np.float64).ctypes.data
        r = self.lib.matel_diag(C.byref(bra), C.byref(ket), ptr)
        return complex(r.re, r.im)

    def exp_diag(self, s: StateT, diag, t: float) -> None:
        if isinstance(diag, int):
            self.lib.exp_diag(C.byref(s), diag, float(t))
            return
        arr = np.ascontiguousarray(diag, dtype=np.float64)
        self.lib.exp_diag(C.byref(s), arr.ctypes.data, float(t))

    def superop(self, kraus) -> np.ndarray:
        ks = np.ascontiguousarray(np.stack([np.asarray(k, dtype=np.complex128) for k in kraus]))
        nq = int(ks.shape[1]).bit_length() - 1
        kt = KrausT(nq, len(kraus), ks.ctypes.data)
        so = self.lib.kraus_to_superop(C.byref(kt))
        m = (ks.shape[1] ** 2)
        raw = (C.c_double * (2 * m * m)).from_address(so.data)
        out = np.frombuffer(raw, dtype=np.complex128, count=m * m).copy().reshape(m, m)
        libc = C.CDLL("libc.so.6")
        libc.free.argtypes = [C.c_void_p]
        libc.free(C.c_void_p(so.data))
        return out

    def channel_1q(self, s: StateT, sop: np.ndarray, q: int) -> None:
        arr = np.ascontiguousarray(np.asarray(sop).reshape(-1), dtype=np.complex128)
        so = SuperopT(1, arr.ctypes.data)
        self.lib.channel_1q(C.byref(s), C.byref(so), int(q))

    def channel_2q(self, s: StateT, sop: np.ndarray, q0: int, q1: int) -> None:
        """2-qubit channel (16 x 16 superoperator, local index 2 bit(q0) + bit(q1))."""
        arr = np.ascontiguousarray(np.asarray(sop).reshape(-1), dtype=np.complex128)
        so = SuperopT(2, arr.ctypes.data)
        self.lib.channel_2q(C.byref(s), C.byref(so), int(q0), int(q1))

    def single_from_mat(self, s: StateT, q: int, mat_colmajor: np.ndarray) -> None:
        arr = np.ascontiguousarray(mat_colmajor, dtype=np.complex128)
        self.lib.single_from_mat(C.byref(s), int(q), arr.ctypes.data)

    def two_from_mat(self, s: StateT, q1: int, q2: int, mat_colmajor: np.ndarray) -> None:
        arr = np.ascontiguousarray(mat_colmajor, dtype=np.complex128)
        self.lib.two_from_mat(C.byref(s), int(q1), int(q2), arr.ctypes.data)

    def sample_matrix(self, iota: StateT, obs, channels, at: int, workspace_bytes: int) -> np.ndarray:
        """S^(at) of include/orkan_sample.h.  channels: a list of (ops, weights), ops Python
        callables op(state: StateT) that apply gates to the state in place, weights a complex
        sequence (None allowed at `at`).  iota is consumed (it holds the prefix state on
        return).  Returns the K x K complex matrix."""
        keep = []
        arr = (SmChannel * len(channels))()
        for k, (ops, weights) in enumerate(channels):
            cbs = [QOP(lambda sp, f=f: f(sp.contents)) for f in ops]
            table = (QOP * len(cbs))(*cbs)
            keep += cbs + [table]
            wptr = None
            if weights is not None:
                w = np.ascontiguousarray(weights, dtype=np.complex128)
                keep.append(w)
                wptr = w.ctypes.data
            arr[k] = SmChannel(len(cbs), C.cast(table, C.POINTER(QOP)), wptr)
        K = len(channels[at][0])
        out = np.zeros((K, K), dtype=np.complex128, order="F")
        ob = obs if isinstance(obs, int) else np.ascontiguousarray(obs, dtype=np.float64)
        self.lib.sample_matrix(C.byref(iota), ob if isinstance(ob, int) else ob.ctypes.data, arr, len(channels),
                               int(at), int(workspace_bytes), out.ctypes.data)
        return out

    def set_stream(self, handle: int | None) -> None:
        self.lib.orkan_set_stream(handle)

    def sync(self) -> None:
        self.lib.orkan_sync()

    def flush(self) -> None:
        """Launch queued statevector gates (see orkan_set_gate_fusion)."""
        self.lib.orkan_flush()

    def set_gate_fusion(self, max_gates: int) -> None:
        self.lib.orkan_set_gate_fusion(int(max_gates))

    def gate_fusion(self) -> int:
        return int(self.lib.orkan_get_gate_fusion())

    def launches(self) -> int:
        return int(self.lib.orkan_launch_count())
