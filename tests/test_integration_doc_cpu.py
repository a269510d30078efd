"""The C examples of INTEGRATION.md compile against include/ldp.h.

The examples are fragments that build on each other (the first declares the
context, parameters, options and job the later ones use), so they are
joined in document order into one function body and compiled with
implicit declarations as errors: a renamed entry point, field or constant
in the header makes this fail.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_c_examples_compile(tmp_path):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```c\n(.*?)```", text, flags=re.S)
    assert len(blocks) >= 3
    body = "\n".join(line for b in blocks for line in b.splitlines() if not line.startswith("#include"))
    src = tmp_path / "examples.c"
    src.write_text('#include "ldp.h"\n#include <stddef.h>\nvoid examples(void) {\n' + body + "\n}\n")
    r = subprocess.run(["gcc", "-std=c11", "-fsyntax-only", "-Wall", "-Werror=implicit-function-declaration",
                        "-Werror=incompatible-pointer-types", "-Wno-unused-variable",
                        "-I", os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_cpp_examples_compile(tmp_path):
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```cpp\n(.*?)```", text, flags=re.S)
    assert blocks
    body = "\n".join(line for b in blocks for line in b.splitlines() if not line.startswith("#include"))
    src = tmp_path / "examples.cpp"
    src.write_text('#include "ldp_engine.hpp"\nint examples(ldp_ctx* ctx, ldp_params p) {\n' + body +
                   "\nreturn 0;\n}\n")
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Wno-unused-variable",
                        "-I", os.path.join(ROOT, "include"), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
