"""The integration examples in tests/examples compile against include/.

tests/examples/integration_example.c holds the C host examples as one
function body; it is compiled with implicit declarations and incompatible
pointer types as errors, so a renamed entry point, field or constant in
include/ldp.h fails here.  tests/examples/integration_example.cpp does the
same for the C++ engine mirror (include/ldp_engine.hpp).
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EX = os.path.join(ROOT, "tests", "examples")


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_examples_compile():
    r = subprocess.run(["gcc", "-std=c11", "-fsyntax-only", "-Wall", "-Werror=implicit-function-declaration",
                        "-Werror=incompatible-pointer-types", "-Wno-unused-variable",
                        "-I", os.path.join(ROOT, "include"), os.path.join(EX, "integration_example.c")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_examples_compile():
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wno-unused-variable",
                        "-I", os.path.join(ROOT, "include"), os.path.join(EX, "integration_example.cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
