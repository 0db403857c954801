"""The host-side plan of the temporally blocked forward passes
(gerjoii_b200/csrc/w_tblock_plan.h) over many grid shapes, depths, tile
shapes and vector widths: every node owned exactly once, streaming tasks
aligned and exact, tiles within their extent, interior tiles free of PML
updates.  Compiled with the host C++ compiler; no GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_blocked_pass_plan_invariants(tmp_path):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "tblock_plan_check"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "gerjoii_b200", "csrc"),
                    os.path.join(ROOT, "tests", "tblock_plan_check.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.startswith("ok "), out.stdout
    assert int(out.stdout.split()[1]) > 1000
