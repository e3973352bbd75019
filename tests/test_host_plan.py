"""The engine's host planning helpers on the CPU (efs_b200/csrc/efs_host.h):
the threaded stable radix sort that orders Mur, TFSF, excitation and RLC
entries by device index, the grouping by target built on it, and the chunked
host-thread loop.  tests/host/host_plan_test.cpp is compiled with g++ against
the same header libefs.so includes and checks them against std::stable_sort
on sorted, reversed, repeated and full-range keys up to 2 M entries."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_host_plan_helpers(tmp_path):
    exe = tmp_path / "host_plan_test"
    src = os.path.join(ROOT, "tests", "host", "host_plan_test.cpp")
    inc = os.path.join(ROOT, "efs_b200", "csrc")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", inc, "-o", str(exe), src], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
