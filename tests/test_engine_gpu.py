"""The C++ mirror of the reference's engine interface (include/ldp_engine.hpp)
returns, trial by trial and lane by lane, the results of the same run
through the job API: Integrate(iTrial) selects trajectory
(rank * NUMBEROFRUNS + iTrial) * lanes + lane of the run.  The object
integrates only its own rank (a job with first_rank = rank), so this also
checks that such a job equals its slice of the whole run bit for bit; its
per-event lists, WRITEX series and range checks are checked too."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import langevindynamicsforpcp_b200 as ldp
from langevindynamicsforpcp_b200 import _lib as L

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "langevindynamicsforpcp_b200")
INP = os.path.join(ROOT, "tests", "golden", "inp", "quick_test__2.0_7.2_m1.0_1.00e-05.inp")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_engine_mirror_matches_the_job_api(tmp_path):
    exe = tmp_path / "engine_check"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "engine_check.cpp"), "-o", str(exe), "-L", LIBDIR, "-lldp",
                    "-Wl,-rpath," + LIBDIR], check=True)
    out = subprocess.run([str(exe), INP, "400000"], capture_output=True, text=True, timeout=300, check=True).stdout
    rows = [l.split() for l in out.splitlines()]
    p = ldp.params_from_inp(INP)
    p.number_of_steps, p.freq_save, p.random_seed = 400000, 200, 1234
    with ldp.Context(0) as ctx, ldp.Job(ctx, p, lanes=8, ranks=2) as j:
        j.run()
        r = j.results(ticks=False)
        means = j.means()
    nr = p.number_of_runs
    nf = r["frames_x"].shape[0]
    assert len(rows) == 8 * nr
    for trial, lane, cnt, fpt, fpt2, tpt, s0, s1, xl, evm, ntpt2, xnan, nv, v0 in rows:
        g = (1 * nr + int(trial)) * 8 + int(lane)
        assert int(cnt) == r["counts"][L.C_FPT][g]
        assert float(fpt) == means[L.E_FPT][g] and float(fpt2) == means[L.E_FPT2][g]
        assert float(tpt) == means[L.E_TPT][g]
        assert float(s0) == r["counts"][L.C_STATE0][g] and float(s1) == r["counts"][L.C_STATE1][g]
        assert float(xl) == r["frames_x"][-1][g]
        # the per-event list, summed in event order, gives the average
        assert float(evm) == (float(fpt) if int(cnt) else -1.0)
        assert int(ntpt2) == r["counts"][L.C_TPT2][g]
        assert xnan == "1"
        assert int(nv) == nf and float(v0) == r["frames_v"][0][g]
    # 40 time units against a mean first-passage time of about 39: events
    assert np.sum(r["counts"][L.C_FPT]) > 0
