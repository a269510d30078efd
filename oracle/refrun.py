"""Runs the CPU-baseline build of the reference's own code (oracle/_ref).

TEST AND CPU-BASELINE INFRASTRUCTURE ONLY: imported by tests/ (statistical
checks of the device paths against the reference's code) and by bench.py's
reference arm and cpu_baseline leg (the reference's CPU path timed on the
host cores).  It imports nothing of the product.

The executables take a .inp file (`-i`); one process is one MPI rank of the
reference with SIMDWIDTH lanes (8 for the AVX-512 build, 4 for AVX2), each
trial NUMBEROFRUNS runs them again.  Processes run in scratch directories
and their output files are read back here.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def exe(model: str = "single", avx512: bool = True) -> str:
    name = "langevinDynamicsSingleBarrier" if model == "single" else "langevinDynamicsDoubleBarrier"
    return os.path.join(REF_DIR, name + ("" if avx512 else "_avx2"))


def available(model: str = "single", avx512: bool = True) -> bool:
    return os.access(exe(model, avx512), os.X_OK)


def lanes(avx512: bool = True) -> int:
    return 8 if avx512 else 4


def inp_text(base_path: str, overrides: dict) -> str:
    """The .inp file at base_path with the keys of `overrides` replaced
    (value: a string, or for FPTCG a list of "flag size" strings that
    replaces every FPTCG line); keys the file lacks are appended."""
    out, seen, cg_done = [], set(), False
    for ln in open(base_path).read().splitlines():
        w = ln.split()
        key = w[0] if w and not w[0].startswith("#") else None
        if key in overrides:
            seen.add(key)
            v = overrides[key]
            if isinstance(v, (list, tuple)):
                if not cg_done:
                    out.extend(f"{key} {e}" for e in v)
                    cg_done = True
                continue
            out.append(f"{key} {v}")
        else:
            out.append(ln)
    for key, v in overrides.items():
        if key not in seen:
            if isinstance(v, (list, tuple)):
                out.extend(f"{key} {e}" for e in v)
            else:
                out.append(f"{key} {v}")
    return "\n".join(out) + "\n"


class Runs:
    """Processes started together, one scratch directory each."""

    def __init__(self, executable: str, inps: list, timeout: float = 600.0):
        self.root = tempfile.mkdtemp(prefix="ldp_ref_")
        self.dirs = []
        procs = []
        t0 = time.perf_counter()
        for i, text in enumerate(inps):
            d = os.path.join(self.root, f"p{i:03d}")
            os.makedirs(d)
            with open(os.path.join(d, "x.inp"), "w") as f:
                f.write(text)
            procs.append(subprocess.Popen([executable, "-i", "x.inp"], cwd=d, stdout=subprocess.DEVNULL,
                                          stderr=subprocess.PIPE))
            self.dirs.append(d)
        self.returncodes, self.errors = [], []
        for p in procs:
            try:
                _, err = p.communicate(timeout=max(1.0, timeout - (time.perf_counter() - t0)))
            except subprocess.TimeoutExpired:
                p.kill()
                _, err = p.communicate()
            self.returncodes.append(p.returncode)
            self.errors.append(err.decode(errors="replace")[-2000:])
        self.wall_s = time.perf_counter() - t0

    def ok(self) -> bool:
        return all(rc == 0 for rc in self.returncodes)

    def path(self, i: int, name: str) -> str:
        return os.path.join(self.dirs[i], name)

    def dat(self, base: str, stat: str) -> np.ndarray:
        """Per-trajectory mean event times of every process, concatenated
        (trial-major, lane-minor within a process, as the reference writes
        <OUTPUTBASE>_<stat>.dat)."""
        return np.concatenate([np.fromfile(self.path(i, f"{base}_{stat}.dat"), dtype="<f8")
                               for i in range(len(self.dirs))])

    def msd(self, base: str, i: int) -> np.ndarray:
        """Process i's MSD curve, rows (time, msd)."""
        return np.loadtxt(self.path(i, f"{base}_msd.log"), comments="#")

    def state_counts(self, base: str, i: int) -> tuple:
        c = [0, 0]
        for ln in open(self.path(i, f"{base}_stateCount.log")):
            w = ln.split()
            if len(w) >= 4 and w[0] == "#" and w[1] == "state":
                c[int(w[2])] = int(w[3])
        return tuple(c)

    def close(self):
        shutil.rmtree(self.root, ignore_errors=True)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
