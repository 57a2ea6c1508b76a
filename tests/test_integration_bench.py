"""The B200 backends for the reference's gate benchmark CLI (orkan_b200/integration/
bench_orkan_b200.c) compile against the reference benchmark's own headers (bench.h vtable,
benchmark/include/bench.h:78-96) with this library's public headers, warnings as errors,
and define both vtables.  Skipped where no copy of the reference is present."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_backends_compile_against_the_reference_benchmark():
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "orkan_b200", "integration"), "check"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    if "no reference benchmark headers" in r.stdout:
        pytest.skip("the reference's benchmark headers are not present")
    assert r.stdout.strip().splitlines()[-1] == "2"          # tiled and packed vtables
