"""The C-ABI libraries load on a machine without a GPU, export every function that
include/*.h declares, and keep the reference's fail-fast validation behaviour
(message "orkan: <module>: <msg>" and exit status 1, reference src/gate/gate.c:19-24,
channel.c:8-13, meas.c:23-28, circ.c:22-27).  No kernel is launched here."""
import ctypes as C
import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")


def declared_functions():
    names = set()
    for f in sorted(os.listdir(INCLUDE)):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(INCLUDE, f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        # expand the backend declaration macro
        m = re.search(r"#define ORKAN_DECLARE_GATE_BACKENDS\(L\)(.*?)\n(?=ORKAN_DECLARE)", text, re.S)
        if m:
            body = m.group(1)
            for layout in ("pure", "packed", "tiled"):
                for g in re.findall(r"void (\w+)_##L\(", body):
                    names.add(f"{g}_{layout}")
            text = text.replace(m.group(0), "")
        text = "\n".join(l for l in text.splitlines()
                          if not l.lstrip().startswith(("#", "ORKAN_DECLARE_GATE_BACKENDS(")))
        for line in text.split(";"):
            line = " ".join(line.split())
            mm = re.match(r"^(?:[\w\s\*]+?)\b(\w+)\s*\([^()]*\)$", line.split("{")[-1].split("}")[-1].strip())
            if mm and not line.startswith(("typedef", "#")):
                names.add(mm.group(1))
    names.discard("ORKAN_DECLARE_GATE_BACKENDS")
    return names


def exported(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


@pytest.mark.parametrize("lt", [5, 3])
def test_library_loads_and_exports_every_declared_symbol(lt):
    from orkan_b200.build import library_path
    path = library_path(lt)
    assert os.path.exists(path), "run __graft_entry__.build() first"
    C.CDLL(path)                                     # loads without a GPU
    decl = declared_functions()
    assert len(decl) > 100                           # public API + backends + C-ABI layer
    missing = decl - exported(path)
    assert not missing, sorted(missing)


def test_public_api_names_match_reference_abi():
    decl = declared_functions()
    for name in ("state_len", "state_init", "state_free", "state_plus", "state_cp", "state_print", "state_get",
                 "state_set", "x", "y", "z", "h", "s", "sdg", "t", "tdg", "hy", "rx", "ry", "rz", "p", "cx", "cy",
                 "cz", "swap_gate", "ccx", "kraus_to_superop", "channel_1q", "mean", "matel_diag", "exp_diag",
                 "x_tiled", "h_packed", "channel_tiled_1q", "mean_tiled", "exp_diag_pure", "single_from_mat",
                 "two_from_mat"):
        assert name in decl, name


PROG = r"""
import ctypes as C, sys
sys.path.insert(0, {root!r})
import orkan_b200
ork = orkan_b200.load(5)
s = orkan_b200.StateT({kind}, C.c_void_p(0x1000), {qubits})
{call}
print("not reached")
"""


def run_child(kind, qubits, call):
    code = PROG.format(root=ROOT, kind=kind, qubits=qubits, call=call)
    return subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("call,msg", [
    ("ork.lib.x(C.byref(s), 5)", "orkan: gate: x: target qubit out of range"),
    ("ork.lib.rx(C.byref(s), 9, 0.3)", "orkan: gate: rx: target qubit out of range"),
    ("ork.lib.cx(C.byref(s), 1, 1)", "orkan: gate: cx: control and target must differ"),
    ("ork.lib.cz(C.byref(s), 7, 1)", "orkan: gate: cz: control qubit out of range"),
    ("ork.lib.swap_gate(C.byref(s), 0, 0)", "orkan: gate: swap: q1 and q2 must differ"),
    ("ork.lib.ccx(C.byref(s), 0, 1, 1)", "orkan: gate: ccx: ctrl2 and target must differ"),
    ("ork.lib.x(None, 0)", "orkan: gate: x: null state or data pointer"),
    ("ork.lib.mean(C.byref(s), None)", "orkan: meas: mean: null observable pointer"),
    ("ork.lib.exp_diag(C.byref(s), None, 1.0)", "orkan: circ: exp_diag: null diagonal pointer"),
])
def test_validation_exits_like_the_reference(call, msg):
    r = run_child(0, 3, call)
    assert r.returncode == 1, r.stderr
    assert msg in r.stderr
    assert "not reached" not in r.stdout


def test_channel_rejects_pure_and_nonlocal():
    call = "so = orkan_b200.SuperopT(1, C.c_void_p(0x2000)); ork.lib.channel_1q(C.byref(s), C.byref(so), 0)"
    r = run_child(0, 3, call)
    assert r.returncode == 1 and "orkan: channel: channel_1q: not available for pure states" in r.stderr
    call = "so = orkan_b200.SuperopT(2, C.c_void_p(0x2000)); ork.lib.channel_1q(C.byref(s), C.byref(so), 0)"
    r = run_child(1, 3, call)
    assert r.returncode == 1 and "orkan: channel: channel_1q: superoperator is not 1-local" in r.stderr


def test_matel_diag_rejects_mixed():
    call = "ork.lib.matel_diag(C.byref(s), C.byref(s), C.c_void_p(0x3000))"
    r = run_child(2, 3, call)
    assert r.returncode == 1 and "orkan: meas: matel_diag: bra must be PURE" in r.stderr


def test_allocation_failure_leaves_null_data():
    """A failed device allocation leaves data == NULL and qubits == 0 with a message, as
    the reference does on host OOM (src/state/state.c:93-97).  The failure is injected on
    the host before any CUDA call."""
    code = f"""
import ctypes as C, sys
sys.path.insert(0, {ROOT!r})
import orkan_b200
ork = orkan_b200.load(5)
ork.lib.orkan_debug_fail_allocs(1)
s = orkan_b200.StateT(0, None, 0)
ork.lib.state_init(C.byref(s), 12, None)
print("data", s.data, "qubits", s.qubits)
"""
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "data None qubits 0" in r.stdout
    assert "state_init(): device allocation failed" in r.stderr


def test_batch_entry_points_declared_and_validate_without_gpu():
    """orkan_batch.h: every entry point is exported, and orkan_qaoa_create rejects invalid
    batches (cudaErrorInvalidValue = 1) before touching a device."""
    from orkan_b200.build import library_path
    decl = declared_functions()
    for f in ("create", "run", "tune", "config", "cost_vector", "stats", "destroy"):
        assert "orkan_qaoa_" + f in decl
    lib = C.CDLL(library_path(5))
    lib.orkan_qaoa_create.argtypes = [C.POINTER(C.c_void_p), C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_uint, C.c_ulonglong, C.c_uint]
    import numpy as np

    def create(ns, edges, offs, p=2):
        ns = np.asarray(ns, np.uint32)
        ed = np.asarray(edges if edges else [0], np.uint32)
        of = np.asarray(offs, np.uint32)
        h = C.c_void_p(1)
        rc = lib.orkan_qaoa_create(C.byref(h), len(ns), ns.ctypes.data, of.ctypes.data, ed.ctypes.data, None, p,
                                   0, 0)
        return rc, h.value

    assert create([27], [], [0, 0]) == (1, None)            # more than 26 qubits
    assert create([0], [], [0, 0]) == (1, None)             # no qubits
    assert create([4], [0, 4], [0, 1]) == (1, None)         # vertex out of range
    assert create([4], [2, 2], [0, 1]) == (1, None)         # self loop
    assert create([4], [0, 1], [0, 1], p=0) == (1, None)    # no layers
    assert create([4, 4], [0, 1], [0, 1, 0]) == (1, None)   # decreasing offsets


def test_state_upload_entry_points_validate_without_gpu():
    """orkan_dev.h: the synchronous and asynchronous uploads and the download reject a null
    state, a state without storage and a null host buffer (cudaErrorInvalidValue = 1) before
    touching a device."""
    from orkan_b200.build import library_path
    decl = declared_functions()
    for f in ("orkan_state_upload", "orkan_state_upload_async", "orkan_state_download"):
        assert f in decl
    lib = C.CDLL(library_path(5))

    class StateT(C.Structure):
        _fields_ = [("type", C.c_int), ("data", C.c_void_p), ("qubits", C.c_ubyte)]

    buf = (C.c_double * 8)()
    empty = StateT(0, None, 1)
    lib.orkan_state_upload_async.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.orkan_state_upload.argtypes = [C.c_void_p, C.c_void_p]
    lib.orkan_state_download.argtypes = [C.c_void_p, C.c_void_p]
    assert lib.orkan_state_upload_async(None, buf, None) == 1
    assert lib.orkan_state_upload_async(C.byref(empty), buf, None) == 1
    assert lib.orkan_state_upload(C.byref(empty), buf) == 1
    assert lib.orkan_state_download(C.byref(empty), buf) == 1
    fake = StateT(0, C.c_void_p(0x1000), 1)
    assert lib.orkan_state_upload_async(C.byref(fake), None, None) == 1
