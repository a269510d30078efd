"""The serving loop's region allocator (csrc/ldp_region.h), on the CPU.

The server allocates its memory budget once and places each admitted job's
arena in it first-fit, merging freed neighbours.  region_check.cpp drives it
with random take/give sequences against a unit-by-unit model: every offset
is the model's first fit, free space is always coalesced into one block per
free run, and the region is whole again once everything is given back.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "langevindynamicsforpcp_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_region_first_fit_and_coalescing(tmp_path):
    exe = tmp_path / "region_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-Wall", "-I", CSRC, os.path.join(HERE, "region_check.cpp"),
                    "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
