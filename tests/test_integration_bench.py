"""The B200 backends for the reference's benchmark CLIs (orkan_b200/integration/
bench_orkan_b200.c): the gate vtable (benchmark/include/bench.h:78-96) and the Kraus vtable
(benchmark/include/bench_kraus.h:54-62) compile against the reference benchmark's own
headers with this library's public headers, warnings as errors; and the reference's own
drivers (bench_main.c, bench_kraus_main.c), linked with these backends under the
reference's backend names, build and start.  Skipped where no copy of the reference is
present (the environment variable ORKAN_REFERENCE_SRC names it)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INTEG = os.path.join(ROOT, "orkan_b200", "integration")


def _make(target):
    r = subprocess.run(["make", "-s", "-C", INTEG, target], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_backends_compile_against_the_reference_benchmark():
    out = _make("check")
    if "no reference benchmark headers" in out:
        pytest.skip("the reference's benchmark headers are not present")
    # gate object: tiled + packed gate vtables; Kraus object: those two + two Kraus vtables
    assert out.strip().splitlines()[-1] == "6"


def test_reference_cli_builds_with_the_b200_backends():
    out = _make("cli")
    if "no reference benchmark sources" in out:
        pytest.skip("the reference's benchmark sources are not present")
    for exe in ("bench_gate_b200", "bench_kraus_b200"):
        path = os.path.join(INTEG, "_build", exe)
        assert os.access(path, os.X_OK)
    r = subprocess.run([os.path.join(INTEG, "_build", "bench_kraus_b200"), "--help"], capture_output=True, text=True)
    assert "--channel" in r.stdout + r.stderr
