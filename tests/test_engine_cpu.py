"""The C++ mirror of the reference's engine interface (include/ldp_engine.hpp)
builds against the library and keeps the reference's error convention on
the CPU: with no device context Integrate returns false after printing the
error, as does a trial past NUMBEROFRUNS; a getter before Integrate prints
an error and returns NaN."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "langevindynamicsforpcp_b200")
INP = os.path.join(ROOT, "tests", "golden", "inp", "quick_test__2.0_7.2_m1.0_1.00e-05.inp")


def build(out):
    subprocess.run(["g++", "-O1", "-std=c++17", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "engine_check.cpp"), "-o", str(out), "-L", LIBDIR, "-lldp",
                    "-Wl,-rpath," + LIBDIR], check=True)


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.exists(os.path.join(LIBDIR, "libldp.so")),
                    reason="no C++ compiler or library not built")
def test_engine_mirror_reports_errors_like_the_reference(tmp_path):
    exe = tmp_path / "engine_check"
    build(exe)
    r = subprocess.run([str(exe), INP, "20000", "nodevice"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.split() == ["0", "0", "1"]
    assert r.stderr.count("Error:") == 3
